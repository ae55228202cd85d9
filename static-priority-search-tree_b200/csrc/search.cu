// Searches of the static priority search tree: one query or a batch of mixed
// 3-sided / 2-sided-left / 2-sided-right queries, in one level-synchronous pass.
//
// The reference walks the tree with one thread block per query, handing subtrees
// to idle threads through shared memory and to child grids when none are idle
// (pst/static-pst-gpu-search-functions.tu:12-722, pst/static-pst-gpu.tu:819-1148).
// Here every query of a batch advances one tree level per kernel (k_bfs_level):
//   - "path" tasks follow the O(log n) boundary nodes of a query with the
//     reference's delegation rules (do3SidedSearchDelegation, doLeftSearchDelegation,
//     doRightSearchDelegation: pst/static-pst-cpu-iter.tpp:602-714);
//   - every subtree the reference would "report above" is scanned by level.  In a
//     max-heap on dim2 a node of such a subtree is reported exactly when its own
//     dim2 passes (its ancestors' dim2 are at least as large), so the work unit is a
//     block: 64 consecutive slots of one level, tested by one warp with coalesced
//     loads.  The frontier is kept as "alive records" only — (block, query, mask of
//     reported slots) — and the next level expands each record into its two child
//     blocks (spread16), masked by occupancy before anything is loaded.  Every
//     level but the last is full (a level-d node holds at least
//     floor((n + 1) / 2^d) - 1 >= 1 points for d <= D - 2), so occupancy is read
//     only for children on the last level.  A block whose whole subtree lies at
//     or above the query's min2 (TreeDev::sub_min) hands its descendants on
//     without any dim2 test (RECORD_WHOLE).
// Small batches start with one CTA that walks the upper levels with its frontier
// in shared memory (k_bfs_cta).  A count of every query falls out of the pass; an
// exclusive scan gives each query's exact output offset, and a flat emit kernel
// writes ids (or points) from the alive records.
#include <algorithm>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda.h>

#include "scan_sort.cuh"
#include "search.cuh"

namespace pst {

namespace {

constexpr uint32_t MODE_THREE = 3, MODE_LEFT = 1, MODE_RIGHT = 2;
constexpr uint32_t FULL = 0xFFFFFFFFu;


template <typename T>
struct QDev {
	const uint32_t *kind;
	const T *min1;
	const T *max1;
	const T *min2;
};

// The same arrays, written once per pass from the caller's pst_query records.
template <typename T>
struct QOut {
	uint32_t *kind;
	T *min1;
	T *max1;
	T *min2;
};

// Alive records cover a "block" of 64 consecutive slots of one level (two
// 128-byte rows of a 4-byte field): (block base position, query, mask of reported
// slots, low and high word).  Block bases are multiples of 64; bit 0 of the first
// word (RECORD_WHOLE) marks a block below which every descendant of the reported
// slots is reported (its dim2 need no test).
constexpr uint32_t RECORD_WHOLE = 1u;

struct WorkDev {
	uint4 *rec;            // alive records of every level, level regions in order
	uint64_t rec_cap;
	uint4 *path0, *path1;  // boundary-path tasks (position, query, mode), double-buffered by level parity
	uint4 *seed0, *seed1;  // report-above seeds (chunk base, query, candidate mask), idem
	uint32_t path_cap;     // entries of each path / seed buffer (2 per query)
	uint4 *ro;             // reported boundary nodes as one-bit block records (never expanded)
	uint32_t ro_cap;
	uint64_t *counts;
	uint64_t *cursor;
	const uint64_t *offsets;
	BatchCtl *ctl;
};

// The block record of a 32-slot chunk (base pos32, a multiple of 32) and its mask.
__device__ __forceinline__ uint4 block_record(uint32_t pos32, uint32_t q, uint32_t bits32)
{
	const bool upper = (pos32 & 32u) != 0;
	return make_uint4(pos32 & ~63u, q, upper ? 0u : bits32, upper ? bits32 : 0u);
}

template <typename T>
__device__ __forceinline__ void path_step(const TreeDev<T> &t, const QDev<T> &qd, const WorkDev &w, uint32_t d,
                                          uint4 task, bool valid)
{
	const uint32_t lane = lane_id();
	const uint32_t h = task.x, q = task.y, mode = task.z;
	const uint32_t l = 2 * h, r = 2 * h + 1;
	const bool inner = d + 1 < t.levels;  // the node has a median and may have children
	bool rep = false;
	uint32_t pl = 0, pr = 0;      // continue as a path task with this mode (0 = no)
	bool rl = false, rr = false;  // report-above subtree
	if (valid) {
		// every value the step may use is loaded at once: one round trip, not a chain.
		// Every level but the last is full, so only children on the last level need
		// their occupancy read.
		const T min2 = qd.min2[q];
		const T v2 = t.dim2[h];
		const uint32_t kind = qd.kind[q];
		const T min1 = qd.min1[q], max1 = qd.max1[q];
		const T v1 = t.dim1[h];
		const uint32_t ow = !inner ? 0u : d + 2 < t.levels ? FULL : t.occ[l >> 5];
		const T m = inner ? t.med[h] : T(0);
		if (min2 <= v2) {
			rep = kind == PST_Q_THREE ? (min1 <= v1 && v1 <= max1) : kind == PST_Q_LEFT ? (v1 <= max1) : (v1 >= min1);
			const bool hl = (ow >> (l & 31)) & 1u, hr = (ow >> (r & 31)) & 1u;
			if (mode == MODE_THREE) {
				if (min1 <= m && m <= max1) {
					pl = hl ? MODE_RIGHT : 0;
					pr = hr ? MODE_LEFT : 0;
				} else if (max1 < m && hl) {
					pl = MODE_THREE;
				} else if (m < min1 && hr) {
					pr = MODE_THREE;
				}
			} else if (mode == MODE_LEFT) {
				if (m <= max1) {
					rl = hl;
					pr = hr ? MODE_LEFT : 0;
				} else if (hl) {
					pl = MODE_LEFT;
				}
			} else {
				if (m >= min1) {
					pl = hl ? MODE_RIGHT : 0;
					rr = hr;
				} else if (hr) {
					pr = MODE_RIGHT;
				}
			}
		}
	}
	// The warp's reported nodes, next-level paths and seeds each take one reservation,
	// and lane 0 issues the three together.  At most two boundary paths per query and
	// level, each leaving at most one seed, so path_cap = 2 * max_q holds every list.
	const bool seed = rl || rr;
	const uint32_t repm = __ballot_sync(FULL, rep);
	const uint32_t seedm = __ballot_sync(FULL, seed);
	const uint32_t npl = (pl ? 1u : 0u) + (pr ? 1u : 0u);
	const uint32_t inc = warp_incl_scan(npl);
	const uint32_t tot = __shfl_sync(FULL, inc, 31);
	uint32_t b_rep = 0, b_path = 0, b_seed = 0;
	if (lane == 0) {
		if (repm)
			b_rep = atomicAdd(&w.ctl->rec_cnt, (uint32_t) __popc(repm));
		if (tot)
			b_path = atomicAdd(&w.ctl->path_cnt[d + 1], tot);
		if (seedm)
			b_seed = atomicAdd(&w.ctl->seed_cnt[d + 1], (uint32_t) __popc(seedm));
	}
	b_rep = __shfl_sync(FULL, b_rep, 0);
	b_path = __shfl_sync(FULL, b_path, 0);
	b_seed = __shfl_sync(FULL, b_seed, 0);
	if (rep) {
		const uint32_t i = b_rep + __popc(repm & lanemask_lt());
		if (i < w.ro_cap)
			w.ro[i] = block_record(h & ~31u, q, 1u << (h & 31));
		else
			atomicOr(&w.ctl->flags, BATCH_FLAG_INTERNAL);
		atomicAdd((unsigned long long *) &w.counts[q], 1ull);
	}
	if (npl) {
		uint32_t i = b_path + inc - npl;
		uint4 *pout = ((d + 1) & 1) ? w.path1 : w.path0;
		if (pl) {
			if (i < w.path_cap)
				pout[i] = make_uint4(l, q, pl, 0);
			else
				atomicOr(&w.ctl->flags, BATCH_FLAG_INTERNAL);
			i++;
		}
		if (pr) {
			if (i < w.path_cap)
				pout[i] = make_uint4(r, q, pr, 0);
			else
				atomicOr(&w.ctl->flags, BATCH_FLAG_INTERNAL);
		}
	}
	if (seed) {
		// l and r share a chunk
		const uint32_t bits = (rl ? 1u << (l & 31) : 0u) | (rr ? 1u << (r & 31) : 0u);
		uint4 *sout = ((d + 1) & 1) ? w.seed1 : w.seed0;
		const uint32_t i = b_seed + __popc(seedm & lanemask_lt());
		if (i < w.path_cap)
			sout[i] = make_uint4(l & ~31u, q, bits, 0u);
		else
			atomicOr(&w.ctl->flags, BATCH_FLAG_INTERNAL);
	}
}

// Appends each lane's non-empty records (at most K) to the level region (one atomic
// per warp).
template <int K>
__device__ __forceinline__ void append_blocks(const WorkDev &w, uint32_t lvl, uint64_t region_base, const uint4 (&r)[K])
{
	const uint32_t lane = lane_id();
	uint32_t nrec = 0;
#pragma unroll
	for (int k = 0; k < K; k++)
		nrec += (r[k].z | r[k].w) ? 1u : 0u;
	const uint32_t inc = warp_incl_scan(nrec);
	const uint32_t tot = __shfl_sync(FULL, inc, 31);
	if (!tot)
		return;
	uint64_t slot0 = 0;
	if (lane == 31) {
		const uint32_t off = atomicAdd(&w.ctl->lvl_cnt[lvl], tot);
		slot0 = region_base + off;
		if (slot0 + tot > w.rec_cap) {
			atomicMax((unsigned long long *) &w.ctl->need_tasks, (unsigned long long) (slot0 + tot));
			atomicOr(&w.ctl->flags, BATCH_FLAG_TASK_OVERFLOW);
			slot0 = ~0ull;
		}
	}
	slot0 = __shfl_sync(FULL, slot0, 31);
	if (slot0 == ~0ull)
		return;
	uint64_t s = slot0 + inc - nrec;
#pragma unroll
	for (int k = 0; k < K; k++)
		if (r[k].z | r[k].w)
			w.rec[s++] = r[k];
}

// Adds the lanes' point counts to their queries' counts (one atomic per run of
// equal query ids).
__device__ __forceinline__ void add_counts(const WorkDev &w, uint32_t q, uint32_t pts, bool valid)
{
	bool last;
	const uint64_t run = warp_run_sum(valid ? q : 0xFFFFFFFFu, pts, &last);
	if (valid && last && run)
		atomicAdd((unsigned long long *) &w.counts[q], (unsigned long long) run);
}

template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
	using V = float4;
};
template <>
struct Vec4<int32_t> {
	using V = int4;
};

// Four consecutive values from a 16-byte aligned address (two loads for doubles).
template <typename T>
__device__ __forceinline__ void load_quad(const T *__restrict__ p, T (&v)[4])
{
	if constexpr (sizeof(T) == 4) {
		using V = typename Vec4<T>::V;
		const V x = *reinterpret_cast<const V *>(p);
		v[0] = x.x;
		v[1] = x.y;
		v[2] = x.z;
		v[3] = x.w;
	} else {
		const double2 a = reinterpret_cast<const double2 *>(p)[0];
		const double2 b = reinterpret_cast<const double2 *>(p)[1];
		v[0] = a.x;
		v[1] = a.y;
		v[2] = b.x;
		v[3] = b.y;
	}
}

// Per-warp shared staging of the 32 records a warp holds: the records, the
// candidate masks of their four child rows (parents' bits spread to their children,
// ANDed with the occupancy), their queries' min2, the child rows found, and the
// list of records that have any candidate at all.
template <typename T>
struct WarpStage {
	uint4 rec[32];
	uint4 cand[32];
	uint4 rows[32];
	T m2[32];
	uint32_t live[32];
};

// Expands the records held by the warp (lane k owns record `mine`; the valid lanes
// are a prefix) into their child records.  Each lane first stages its record's
// candidate child slots (`full`: the children's level is full, so the candidates
// are the spread parent bits with no occupancy read); records without any (all
// children absent, e.g. above a sparse last level) cost nothing more.  Then the whole warp takes the live records
// U at a time: lane l tests the child slots [2b + 4l, 2b + 4l + 4) with one 16-byte
// load (two for doubles), issued only where it has candidates; each 8-lane group
// ORs its nibbles into one 32-slot child row, and the owner reads the four rows as
// its two child records (blocks 2b and 2b + 64).
template <typename T, bool LAST>
__device__ __forceinline__ void expand_records(const TreeDev<T> &t, const T *__restrict__ min2s, const uint4 &mine,
                                               bool valid, bool full, WarpStage<T> &st, uint4 (&child)[2],
                                               uint32_t &pts)
{
	constexpr int U = sizeof(T) == 4 ? 4 : 2;  // records in flight
	const uint32_t lane = lane_id();
	const uint32_t r = lane >> 3, qd = lane & 7;
	const uint32_t base = mine.x & ~63u;  // bit 0 of a record's block: RECORD_WHOLE
	// the record's min2 stays in its owner lane's register (its load overlaps the
	// staging below) and is broadcast by a shuffle where it is compared
	const T m2_own = valid ? min2s[mine.y] : T(0);
	// A block whose every descendant has dim2 >= min2 (TreeDev::sub_min): all
	// descendants of its reported slots are reported, with no test; its child
	// records carry RECORD_WHOLE, so theirs need no look-up either.
	bool whole = (mine.x & RECORD_WHOLE) != 0;
	if (valid && !whole && t.sub_min && base >= 64)
		whole = m2_own <= t.sub_min[base >> 6];
	uint4 cand = make_uint4(0, 0, 0, 0);
	bool has_children = valid;
	if (LAST && valid) {
		// expanding into the last level: most blocks of a sparse last level have no
		// children, which one bit per parent block tells before any occupancy read
		const uint32_t j = (base - (1u << (t.levels - 2))) >> 6;
		has_children = (t.last_par[j >> 5] >> (j & 31)) & 1u;
	}
	if (has_children) {
		// children on a full level (every level but the last) need no occupancy read
		const uint4 occ = full ? make_uint4(FULL, FULL, FULL, FULL)
		                       : *reinterpret_cast<const uint4 *>(t.occ + ((2 * base) >> 5));
		cand = make_uint4(spread16(mine.z) & occ.x, spread16(mine.z >> 16) & occ.y, spread16(mine.w) & occ.z,
		                  spread16(mine.w >> 16) & occ.w);
	}
	const bool live = !whole && (cand.x | cand.y | cand.z | cand.w) != 0;
	const uint32_t lm = __ballot_sync(FULL, live);
	const int nlive = __popc(lm);
	if (live) {
		st.rec[lane] = mine;
		st.cand[lane] = cand;
		st.live[__popc(lm & lanemask_lt())] = lane;
	}
	__syncwarp();
	const uint32_t *candw = reinterpret_cast<const uint32_t *>(st.cand);
	for (int k0 = 0; k0 < nlive; k0 += U) {
		uint32_t cn[U], kk[U];
		T v[U][4];
#pragma unroll
		for (int u = 0; u < U; u++) {
			const bool on = k0 + u < nlive;
			const uint32_t k = st.live[on ? k0 + u : 0];
			kk[u] = k;
			const uint32_t c4 = on ? (candw[4 * k + r] >> (4 * qd)) & 0xFu : 0u;
			cn[u] = c4;
			if (c4) {
				load_quad(t.dim2 + 2 * (st.rec[k].x & ~63u) + 4 * lane, v[u]);
			} else {
#pragma unroll
				for (int j = 0; j < 4; j++)
					v[u][j] = T(0);
			}
		}
#pragma unroll
		for (int u = 0; u < U; u++) {
			const T m2 = __shfl_sync(FULL, m2_own, kk[u]);
			// all four slots are compared (values of slots without a candidate are zero or
			// loaded anyway) and the candidates masked once, not tested slot by slot
			uint32_t ge = 0;
#pragma unroll
			for (int j = 0; j < 4; j++)
				ge |= (m2 <= v[u][j]) ? 1u << j : 0u;
			uint32_t row = (ge & cn[u]) << (4 * qd);
			row |= __shfl_xor_sync(FULL, row, 1);
			row |= __shfl_xor_sync(FULL, row, 2);
			row |= __shfl_xor_sync(FULL, row, 4);
			if (qd == 0 && k0 + u < nlive)
				reinterpret_cast<uint32_t *>(st.rows)[4 * kk[u] + r] = row;
		}
	}
	__syncwarp();
	// the tested rows, or for a whole block its candidates (all reported)
	const uint4 rw = live ? st.rows[lane] : whole ? cand : make_uint4(0, 0, 0, 0);
	const uint32_t cx = 2 * base + (whole ? RECORD_WHOLE : 0u);
	child[0] = make_uint4(cx, mine.y, rw.x, rw.y);
	child[1] = make_uint4(cx + 64, mine.y, rw.z, rw.w);
	pts = __popc(rw.x) + __popc(rw.y) + __popc(rw.z) + __popc(rw.w);
	__syncwarp();  // the stage is reused by the warp's next batch
}

// One tree level of the search (the body of k_bfs_level): the boundary paths, the
// seeds and the expansion of the previous level's records, spread over `gwarps`
// warps (of the grid, or of the one CTA of k_bfs_cta).
// cnt: the level's boundary-path tasks and seeds (ctl->path_cnt[d], seed_cnt[d]
// capped at path_cap) in shared memory, read by the caller with the level's other
// counters.
template <typename T, bool LAST>
__device__ __forceinline__ void level_body(const TreeDev<T> &t, const QDev<T> &qd, const WorkDev &w, uint32_t d,
                                           uint64_t gwarp, uint64_t gwarps, uint64_t base_prev, uint64_t base_cur,
                                           uint64_t n_prev, const uint32_t *cnt, WarpStage<T> &stage)
{
	const uint32_t lane = lane_id();
	const uint32_t np = cnt[0], ns = cnt[1];
	// The level's three kinds of work go to disjoint sets of warps so that their
	// dependent-load chains overlap instead of adding up: a few warps take the
	// boundary paths, a few the seeds, the rest the records.
	const uint64_t cap = gwarps / 8 + 1;
	const uint64_t wp = min((uint64_t) (np + 31) / 32, cap);
	const uint64_t ws = min((uint64_t) (ns + 31) / 32, cap);
	const uint64_t wr = gwarps - wp - ws;  // >= 1: the grid has at least 4 warps

	if (gwarp < wp) {
		// boundary paths, one task per lane
		const uint4 *pin = (d & 1) ? w.path1 : w.path0;
		for (uint64_t wb = gwarp * 32; wb < np; wb += wp * 32) {
			const bool valid = wb + lane < np;
			path_step<T>(t, qd, w, d, valid ? pin[wb + lane] : make_uint4(0, 0, 0, 0), valid);
		}
	} else if (gwarp < wp + ws) {
		// report-above seeds of this level: one or two candidate slots each, tested
		// by their own lane
		const uint4 *sin = (d & 1) ? w.seed1 : w.seed0;
		for (uint64_t wb = (gwarp - wp) * 32; wb < ns; wb += ws * 32) {
			const bool valid = wb + lane < ns;
			const uint4 sd = valid ? sin[wb + lane] : make_uint4(0, 0, 0, 0);
			uint32_t am = 0;
			if (sd.z) {
				// a seed's candidates are the two children of one node, an aligned pair of
				// slots: their dim2, the occupancy (read on the last level only, all
				// others being full) and min2 come in one round trip
				const uint32_t p = (__ffs(sd.z) - 1) & ~1u;
				const uint32_t cand = sd.z & (d + 1 < t.levels ? FULL : t.occ[sd.x >> 5]);
				const T m2 = qd.min2[sd.y];
				T v[2];
				if constexpr (sizeof(T) == 4) {
					const uint2 x = *reinterpret_cast<const uint2 *>(t.dim2 + sd.x + p);
					memcpy(&v[0], &x.x, 4);
					memcpy(&v[1], &x.y, 4);
				} else {
					const double2 x = *reinterpret_cast<const double2 *>(t.dim2 + sd.x + p);
					v[0] = x.x;
					v[1] = x.y;
				}
#pragma unroll
				for (int j = 0; j < 2; j++)
					am |= (((cand >> (p + j)) & 1u) && m2 <= v[j]) ? 1u << (p + j) : 0u;
			}
			add_counts(w, sd.y, __popc(am), valid);
			const uint4 one[1] = {am ? block_record(sd.x, sd.y, am) : make_uint4(0, 0, 0, 0)};
			append_blocks<1>(w, d, base_cur, one);
		}
	} else {
		// expansion of the previous level's alive records into their child blocks, 32
		// consecutive records per warp (their children stay together in the next
		// level's region, which keeps that level's chunks local)
		// A narrow level (records fewer than a quarter of the record warps' lanes)
		// gives each warp 8 consecutive records instead of 32: four times the warps
		// work on it, each with a quarter of the dependent load rounds, and the
		// children of 8 consecutive parents still stay together in the next level.
		const uint64_t per = n_prev * 4 < wr * 32 ? 8 : 32;
		uint64_t wb = (gwarp - wp - ws) * per;
		bool nvalid = lane < per && wb + lane < n_prev;
		uint4 nxt = nvalid ? w.rec[base_prev + wb + lane] : make_uint4(0, 0, 0, 0);
		// A round's children are reserved with one atomic per warp, but written in the
		// next round, after that round's loads: the reservation's latency overlaps them.
		// Pending: this lane's first child block (the second at pp + 64), query, the
		// four child mask words, its first slot offset in the warp's run, and the
		// warp's reservation (lane 31; ~0 = none or refused).
		uint32_t pp = 0, pq = 0, pofs = 0, pres = ~0u;
		uint4 pm = make_uint4(0, 0, 0, 0);
		auto flush = [&]() {
			const uint32_t r0 = __shfl_sync(FULL, pres, 31);
			if (r0 == ~0u)
				return;
			uint64_t sl = base_cur + r0 + pofs;
			if (pm.x | pm.y)
				w.rec[sl++] = make_uint4(pp, pq, pm.x, pm.y);
			if (pm.z | pm.w)
				w.rec[sl] = make_uint4(pp + 64, pq, pm.z, pm.w);
		};
		for (; wb < n_prev; wb += wr * per) {
			const bool valid = nvalid;
			const uint4 mine = nxt;
			// the next round's record is read now, its load overlapping this round
			const uint64_t nb = wb + wr * per;
			nvalid = lane < per && nb + lane < n_prev;
			nxt = nvalid ? w.rec[base_prev + nb + lane] : make_uint4(0, 0, 0, 0);
			uint4 child[2];
			uint32_t pts;
			expand_records<T, LAST>(t, qd.min2, mine, valid, !LAST && d + 1 < t.levels, stage,
			                        child, pts);
			// a warp whose records found no child (most of them when a sparse last
			// level is expanded) has nothing to count or append
			if (__ballot_sync(FULL, pts != 0) == 0)
				continue;
			add_counts(w, mine.y, pts, valid);
			flush();
			const uint32_t nrec = ((child[0].z | child[0].w) ? 1u : 0u) + ((child[1].z | child[1].w) ? 1u : 0u);
			const uint32_t inc = warp_incl_scan(nrec);
			pres = ~0u;
			if (lane == 31) {
				// inc = the warp's total here (pts != 0 somewhere, so it is positive)
				const uint32_t off = atomicAdd(&w.ctl->lvl_cnt[d], inc);
				if (base_cur + off + inc > w.rec_cap) {
					atomicMax((unsigned long long *) &w.ctl->need_tasks, (unsigned long long) (base_cur + off + inc));
					atomicOr(&w.ctl->flags, BATCH_FLAG_TASK_OVERFLOW);
				} else {
					pres = off;
				}
			}
			pp = child[0].x;
			pq = mine.y;
			pofs = inc - nrec;
			pm = make_uint4(child[0].z, child[0].w, child[1].z, child[1].w);
		}
		flush();
	}
}

// LAST: the expansion into the last level of a tree with TreeDev::last_par (its own
// instantiation, so the other levels keep their register budget).  THREADS: the
// CTA size (128, 256 or 512, a tuning choice); every size keeps 64 registers a
// thread, so 1024 threads of the kernel fit an SM at once.
template <typename T, bool LAST, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_bfs_level(TreeDev<T> t, QDev<T> qd, WorkDev w,
                                                                      uint32_t d)
{
	// Launched as a programmatic dependent of the previous level: its CTAs may be
	// scheduled while that level drains, and wait here until it has completed and
	// its writes are visible (a no-op for an ordinary launch).
	asm volatile("griddepcontrol.wait;" ::: "memory");
	__shared__ uint64_t s_base[2];
	__shared__ uint32_t s_cnt[3];  // paths, seeds, stop
	__shared__ WarpStage<T> s_stage[THREADS / 32];
	if (threadIdx.x == 0) {
		// the level's counters, all in one round trip: the previous region's start and
		// length, this level's paths and seeds, and the flags
		const uint64_t b = d ? w.ctl->lvl_base[d - 1] : 0;
		const uint32_t c = d ? w.ctl->lvl_cnt[d - 1] : 0u;
		const uint32_t np = w.ctl->path_cnt[d], ns = w.ctl->seed_cnt[d], fl = w.ctl->flags;
		s_base[0] = b;
		s_base[1] = b + c;
		s_cnt[0] = min(np, w.path_cap);
		s_cnt[1] = min(ns, w.path_cap);
		s_cnt[2] = fl & BATCH_FLAG_TASK_OVERFLOW;
		if (blockIdx.x == 0)
			w.ctl->lvl_base[d] = b + c;
	}
	__syncthreads();
	// Once the frontier has overflowed, the reservation that crossed the capacity
	// left some slots below it unwritten, so nothing of the previous level may be
	// read: the pass stops here and the host repeats it with a larger buffer.
	if (s_cnt[2])
		return;
	const uint64_t base_prev = s_base[0], base_cur = s_base[1];
	// after a frontier overflow the counters run past what was stored: never read beyond it
	const uint64_t end_prev = min(base_cur, w.rec_cap);
	const uint64_t n_prev = end_prev > base_prev ? end_prev - base_prev : 0;
	const uint64_t gthreads = (uint64_t) gridDim.x * blockDim.x;
	const uint64_t gtid = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
	const uint64_t gwarps = gthreads / 32, gwarp = gtid / 32;
	level_body<T, LAST>(t, qd, w, d, gwarp, gwarps, base_prev, base_cur, n_prev, s_cnt,
	                    s_stage[threadIdx.x >> 5]);
}

// Query i of the batch: its kind and bounds into the engine's per-query arrays, and
// its level-0 boundary path task (returned); a kind out of range raises
// BATCH_FLAG_BAD_QUERY in *flags (the pass still runs, and the host reports it).
template <typename T>
__device__ __forceinline__ uint4 unpack_query(const pst_query *__restrict__ raw, uint32_t i, const QOut<T> &qo,
                                              uint32_t *flags)
{
	const pst_query q = raw[i];
	T a, b, c;
	if constexpr (sizeof(T) == 8) {
		a = q.min1.f64; b = q.max1.f64; c = q.min2.f64;
	} else if constexpr (std::is_same<T, float>::value) {
		a = q.min1.f32; b = q.max1.f32; c = q.min2.f32;
	} else {
		a = q.min1.i32; b = q.max1.i32; c = q.min2.i32;
	}
	const int32_t k = q.kind;
	if (k < PST_Q_THREE || k > PST_Q_RIGHT)
		atomicOr(flags, BATCH_FLAG_BAD_QUERY);
	qo.kind[i] = (uint32_t) k;
	qo.min1[i] = a;
	qo.max1[i] = b;
	qo.min2[i] = c;
	const uint32_t mode = k == PST_Q_THREE ? MODE_THREE : k == PST_Q_LEFT ? MODE_LEFT : MODE_RIGHT;
	return make_uint4(1u, i, mode, 0u);
}

// The pass's control block from the engine's pinned host copy, read through its
// mapped device address: a kernel, because inside the captured pass a
// host-to-device copy node ahead of the first kernel left the device idle for
// ≈ 25 µs per pass.
__global__ void k_load_ctl(const BatchCtl *src, BatchCtl *dst)
{
	const uint32_t *s = reinterpret_cast<const uint32_t *>(src);
	uint32_t *d = reinterpret_cast<uint32_t *>(dst);
	for (uint32_t i = threadIdx.x; i < sizeof(BatchCtl) / 4; i += blockDim.x)
		d[i] = s[i];
}

// Start of a full pass (after the control block's load): the batch's queries
// unpacked and checked, their level-0 paths, and the per-query counts and output
// cursors zeroed (all max_q of them: the scan reads every count).
template <typename T>
__global__ void k_prepare_queries(const pst_query *raw, BatchCtl *ctl, QOut<T> qo, uint4 *path0, uint64_t *counts,
                                  uint64_t *cursor, uint32_t max_q)
{
	const uint32_t nq = ctl->nq;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < max_q; i += gridDim.x * blockDim.x) {
		if (i < nq)
			path0[i] = unpack_query<T>(raw, i, qo, &ctl->flags);
		counts[i] = 0;
		cursor[i] = 0;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0)
		ctl->path_cnt[0] = nq;
}

// Small batches (a single query, or a few): one CTA takes the tree from the top,
// level by level with a CTA barrier in place of a kernel boundary, while the
// records to expand stay few enough for it (at most CTA_REC_CAP); it leaves
// ctl->cta_levels = the levels done and the host launches the per-level kernels
// for the rest only.  When it reaches the bottom it also scans the queries'
// counts into offsets[0..max_q] and total, so no scan pass is needed.
//
// The pass works in shared memory: the control block, the boundary paths and
// seeds (pcap of each of the four lists) and the alive records of every level it
// takes (rcap) live in the dynamic shared array, so a level waits on its tree
// loads alone, not on round trips to L2 for its counters, records and
// reservations.  Where it stops, it writes the records, the control block and the
// next level's paths and seeds to their global buffers, in the layout the
// per-level kernels and the emit read.  It stops early when the next level might
// not fit in rcap.
constexpr uint32_t CTA_REC_CAP = 256;

// Dynamic shared memory of k_bfs_cta: the control block, then the four path and
// seed lists, then the records.
__host__ __device__ constexpr size_t cta_smem_bytes(uint32_t pcap, uint32_t rcap)
{
	return sizeof(BatchCtl) + (size_t) (4 * pcap + rcap) * sizeof(uint4);
}
static_assert(sizeof(BatchCtl) % 16 == 0, "the lists after the control block stay 16-byte aligned");

template <typename T>
__global__ void __launch_bounds__(BFS_THREADS, 1) k_bfs_cta(TreeDev<T> t, QDev<T> qd, WorkDev wg, uint32_t max_q,
                                                            uint32_t pcap, uint32_t rcap, const pst_query *raw,
                                                            QOut<T> qo, const BatchCtl *ctl_src)
{
	extern __shared__ __align__(16) unsigned char s_dyn[];
	__shared__ WarpStage<T> s_stage[BFS_THREADS / 32];
	__shared__ uint64_t s_base[2];
	__shared__ uint64_t s_wsum[BFS_THREADS / 32];
	__shared__ uint32_t s_go, s_cnt[2];
	BatchCtl *sc = reinterpret_cast<BatchCtl *>(s_dyn);
	uint4 *sl = reinterpret_cast<uint4 *>(s_dyn + sizeof(BatchCtl));
	// the shared-memory view of the work buffers (ids of reported boundary nodes,
	// counts and offsets stay global)
	WorkDev w = wg;
	w.ctl = sc;
	w.path0 = sl;
	w.path1 = sl + pcap;
	w.seed0 = sl + 2 * pcap;
	w.seed1 = sl + 3 * pcap;
	w.path_cap = pcap;
	w.rec = sl + 4 * pcap;
	w.rec_cap = rcap;
	{
		// the pass's starting control block: the engine's pinned host copy (or the
		// no-alloc search's device copy), wg.ctl receives the final one
		const uint32_t *src = reinterpret_cast<const uint32_t *>(ctl_src);
		uint32_t *dst = reinterpret_cast<uint32_t *>(sc);
		for (uint32_t i = threadIdx.x; i < sizeof(BatchCtl) / 4; i += BFS_THREADS)
			dst[i] = src[i];
	}
	__syncthreads();
	{
		// the start of the pass (k_prepare_queries of a full pass): the queries
		// unpacked and checked, their level-0 paths (at most pcap / 2 queries: the
		// host runs this pass for small batches only), the counts and cursors zeroed
		const uint32_t nq = min(sc->nq, pcap);
		for (uint32_t i = threadIdx.x; i < max_q; i += BFS_THREADS) {
			if (i < nq)
				w.path0[i] = unpack_query<T>(raw, i, qo, &sc->flags);
			wg.counts[i] = 0;
			wg.cursor[i] = 0;
		}
		if (threadIdx.x == 0)
			sc->path_cnt[0] = nq;
	}
	__syncthreads();
	const uint64_t gwarps = BFS_THREADS / 32, gwarp = threadIdx.x >> 5;
	uint64_t acc_prev = 0, acc = 0;  // (thread 0) start of the previous level's records, and of this level's
	uint32_t d = 0;
	for (; d < t.levels; d++) {
		if (threadIdx.x == 0) {
			const uint32_t prev = d ? sc->lvl_cnt[d - 1] : 0u;
			const uint32_t np = min(sc->path_cnt[d], pcap), ns = min(sc->seed_cnt[d], pcap);
			if (d) {
				acc_prev = acc;
				acc += prev;
			}
			s_base[0] = acc_prev;
			s_base[1] = acc;
			s_cnt[0] = np;
			s_cnt[1] = ns;
			// the level appends at most two children per record and one record per seed
			s_go = !(sc->flags & BATCH_FLAG_TASK_OVERFLOW) && prev <= CTA_REC_CAP &&
			       acc + 2 * (uint64_t) prev + ns <= rcap;
			if (s_go)
				sc->lvl_base[d] = acc;
		}
		__syncthreads();
		if (!s_go)
			break;
		const uint64_t base_prev = s_base[0], base_cur = s_base[1];
		const uint64_t n_prev = base_cur - base_prev;
		if (d + 1 == t.levels && t.last_par)
			level_body<T, true>(t, qd, w, d, gwarp, gwarps, base_prev, base_cur, n_prev, s_cnt, s_stage[gwarp]);
		else
			level_body<T, false>(t, qd, w, d, gwarp, gwarps, base_prev, base_cur, n_prev, s_cnt, s_stage[gwarp]);
		__syncthreads();  // the level's records, paths, seeds and counts are visible to the CTA
		if (threadIdx.x == 0)
			sc->cta_levels = d + 1;
	}
	// Hand over: the records of the levels taken (acc of them, levels 0..d-1), and,
	// where the pass stopped above the bottom, the paths and seeds of level d.
	if (threadIdx.x == 0) {
		// records written: at the bottom, acc is the start of the last level's region
		// and that level's count follows it; where the pass stopped at level d, the
		// top of the loop had already advanced acc past level d - 1, so acc is the
		// number written (at most rcap in both cases: each level's bound was checked
		// before it ran)
		const uint64_t n = d == t.levels && d ? acc + sc->lvl_cnt[d - 1] : acc;
		// (a refused reservation, which the bound rules out, would have raised the
		// overflow flag and left the counts past what was stored: never copy beyond)
		s_base[0] = min(n, (uint64_t) rcap);
		if (n > wg.rec_cap) {
			sc->need_tasks = max((unsigned long long) sc->need_tasks, (unsigned long long) n);
			sc->flags |= BATCH_FLAG_TASK_OVERFLOW;
		}
		s_go = d == t.levels && !(sc->flags & BATCH_FLAG_TASK_OVERFLOW);
	}
	__syncthreads();
	{
		const uint64_t n = s_base[0];
		if (n <= wg.rec_cap)
			for (uint64_t i = threadIdx.x; i < n; i += BFS_THREADS)
				wg.rec[i] = w.rec[i];
		if (d < t.levels) {
			const uint32_t np = min(sc->path_cnt[d], pcap), ns = min(sc->seed_cnt[d], pcap);
			const uint4 *ps = (d & 1) ? w.path1 : w.path0, *ss = (d & 1) ? w.seed1 : w.seed0;
			uint4 *pd = (d & 1) ? wg.path1 : wg.path0, *sd = (d & 1) ? wg.seed1 : wg.seed0;
			for (uint32_t i = threadIdx.x; i < np; i += BFS_THREADS)
				pd[i] = ps[i];
			for (uint32_t i = threadIdx.x; i < ns; i += BFS_THREADS)
				sd[i] = ss[i];
		}
	}
	if (s_go) {
		// exclusive scan of counts[0..max_q) in chunks of one count per thread
		const uint32_t nq = sc->nq, lane = lane_id();
		uint64_t *offsets = const_cast<uint64_t *>(w.offsets);
		uint64_t carry = 0;
		for (uint32_t b = 0; b < max_q; b += BFS_THREADS) {
			const uint32_t q = b + threadIdx.x;
			const uint64_t c = q < nq ? w.counts[q] : 0;
			const uint64_t inc = warp_incl_scan(c);
			if (lane == 31)
				s_wsum[gwarp] = inc;
			__syncthreads();
			if (gwarp == 0) {
				uint64_t v = lane < BFS_THREADS / 32 ? s_wsum[lane] : 0;
				v = warp_incl_scan(v);
				if (lane < BFS_THREADS / 32)
					s_wsum[lane] = v;
			}
			__syncthreads();
			if (q < max_q)
				offsets[q] = carry + (gwarp ? s_wsum[gwarp - 1] : 0) + inc - c;
			carry += s_wsum[BFS_THREADS / 32 - 1];
			__syncthreads();  // s_wsum is rewritten by the next chunk
		}
		if (threadIdx.x == 0) {
			offsets[max_q] = carry;
			sc->total = carry;
		}
	}
	__syncthreads();
	// the control block last: every counter the host and the next kernels read
	{
		const uint32_t *src = reinterpret_cast<const uint32_t *>(sc);
		uint32_t *dst = reinterpret_cast<uint32_t *>(wg.ctl);
		for (uint32_t i = threadIdx.x; i < sizeof(BatchCtl) / 4; i += BFS_THREADS)
			dst[i] = src[i];
	}
}

// Shared memory the one-CTA top pass may take beyond its static arrays on the
// current device, after allowing it for the kernel there (once per device; done
// before any launch is captured into a graph).
template <typename T>
size_t cta_pass_budget()
{
	static std::mutex mu;
	static size_t budget[64];
	static bool done[64] = {};
	const DeviceInfo &di = device_info();
	std::lock_guard<std::mutex> lk(mu);
	if (!done[di.device]) {
		cudaFuncAttributes a{};
		PST_CUDA(cudaFuncGetAttributes(&a, k_bfs_cta<T>));
		const size_t b = di.smem_optin > a.sharedSizeBytes + 1024 ? di.smem_optin - a.sharedSizeBytes - 1024 : 0;
		PST_CUDA(cudaFuncSetAttribute(k_bfs_cta<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) b));
		budget[di.device] = b;
		done[di.device] = true;
	}
	return budget[di.device];
}

// Launches the one-CTA top pass with its shared-memory lists: pcap entries for each
// path and seed list (at least two per query of the batch) and as many records as
// the rest of the CTA's shared memory holds.
template <typename T>
void launch_cta_pass(const TreeDev<T> &tv, const QDev<T> &qd, const WorkDev &w, uint32_t max_q, uint32_t pcap,
                     const pst_query *raw, const QOut<T> &qo, const BatchCtl *ctl_src, cudaStream_t s)
{
	const size_t budget = cta_pass_budget<T>();
	const size_t fixed = cta_smem_bytes(pcap, 0);
	// room for at least one level's records beyond the lists
	if (budget < fixed + (size_t) (2 * CTA_REC_CAP + pcap) * sizeof(uint4))
		fail(PST_ERR_INTERNAL, "shared memory too small for the top pass of " + std::to_string(max_q) + " queries");
	const uint32_t rcap = (uint32_t) ((budget - fixed) / sizeof(uint4));
	k_bfs_cta<T><<<1, BFS_THREADS, cta_smem_bytes(pcap, rcap), s>>>(tv, qd, w, max_q, pcap, rcap, raw, qo,
	                                                                  ctl_src);
}

// Output slot of this lane's record inside its query's result: one atomic per run
// of equal query ids on the query's cursor.
__device__ __forceinline__ uint64_t claim_output(const WorkDev &w, uint32_t q, uint32_t pc, bool valid)
{
	bool last;
	const uint64_t run = warp_run_sum(valid ? q : 0xFFFFFFFFu, pc, &last);
	const uint32_t lastmask = __ballot_sync(FULL, last);
	const uint32_t run_last = (uint32_t) (__ffs(lastmask & (FULL << lane_id())) - 1);
	uint64_t rb = 0;
	if (valid && last && run)
		rb = atomicAdd((unsigned long long *) &w.cursor[q], (unsigned long long) run);
	rb = __shfl_sync(FULL, rb, run_last);
	return (valid && pc) ? w.offsets[q] + rb + run - pc : 0;
}

// Output range check of one lane's record, made once where the lane claims it: a
// record whose claimed range would end past the output's capacity is cleared (it
// writes nothing) and flagged.  Counts and claims come from the same masks, so this
// never fires; it keeps the warp-wide store loop of emit_blocks free of per-store
// checks (a 64-bit compare at every 4-byte store cost 8 % of a batched step).
__device__ __forceinline__ void guard_claim(const WorkDev &w, uint4 &rec, uint64_t out_base, uint64_t capacity)
{
	if (out_base + __popc(rec.z) + __popc(rec.w) > capacity) {
		atomicOr(&w.ctl->flags, BATCH_FLAG_INTERNAL);
		rec.z = rec.w = 0;
	}
}

// Writes the results of the warp's records (lane k owns record `mine`, whose results
// start at out_base, checked by guard_claim; the valid lanes are a prefix): the
// lanes stage their records and offsets, then the warp writes U records at a time,
// each by the whole warp, lane l taking slots 2l and 2l + 1 of the 64-slot block.
struct EmitStage {
	uint4 rec[32];
	unsigned long long ob[32];
};

template <typename T, bool HAS_ID, bool POINTS, int U>
__device__ __forceinline__ void emit_blocks(const TreeDev<T> &t, const uint4 &mine, uint64_t out_base, bool valid,
                                            EmitStage &st, void *__restrict__ out)
{
	using Pt = Point<T, HAS_ID>;  // U: records in flight per warp
	static_assert(32 % U == 0, "a batch of records ends inside the 32 staged ones");
	const uint32_t lane = lane_id();
	const uint32_t psh = (2 * lane) & 31;
	// the record's slots before this lane's pair, as masks of its two 32-slot words
	const uint32_t below_z = lane < 16 ? (1u << psh) - 1u : FULL;
	const uint32_t below_w = lane < 16 ? 0u : (1u << psh) - 1u;
	st.rec[lane] = mine;
	st.ob[lane] = out_base;
	__syncwarp();
	const int nrec = __popc(__ballot_sync(FULL, valid));
	for (int k0 = 0; k0 < nrec; k0 += U) {
		uint32_t b2[U], hb[U];
		uint64_t o[U];
		uint2 idv[U];
		T d1[POINTS ? U : 1][2], d2[POINTS ? U : 1][2];
#pragma unroll
		for (int u = 0; u < U; u++) {
			// every lane staged a record, and those past nrec are empty (zero masks), so
			// a batch that runs past nrec reads them and writes nothing: no bound test
			// per record (U divides 32, so k < 32)
			const int k = k0 + u;
			const uint4 rc = st.rec[k];
			b2[u] = ((lane < 16 ? rc.z : rc.w) >> psh) & 3u;
			const uint32_t before = __popc(rc.z & below_z) + __popc(rc.w & below_w);
			o[u] = st.ob[k] + before;
			hb[u] = (rc.x & ~63u) + 2 * lane;  // (without RECORD_WHOLE)
			if constexpr (!POINTS || HAS_ID)
				idv[u] = b2[u] ? *reinterpret_cast<const uint2 *>(t.id + hb[u]) : make_uint2(0, 0);
			if constexpr (POINTS) {
				// the slot pair's dim1 and dim2 with one 8-byte (16 for doubles) load each
				d1[u][0] = d1[u][1] = d2[u][0] = d2[u][1] = T(0);
				if (b2[u]) {
					if constexpr (sizeof(T) == 4) {
						const uint2 a = *reinterpret_cast<const uint2 *>(t.dim1 + hb[u]);
						const uint2 c = *reinterpret_cast<const uint2 *>(t.dim2 + hb[u]);
						memcpy(&d1[u][0], &a.x, 4);
						memcpy(&d1[u][1], &a.y, 4);
						memcpy(&d2[u][0], &c.x, 4);
						memcpy(&d2[u][1], &c.y, 4);
					} else {
						const double2 a = *reinterpret_cast<const double2 *>(t.dim1 + hb[u]);
						const double2 c = *reinterpret_cast<const double2 *>(t.dim2 + hb[u]);
						d1[u][0] = a.x;
						d1[u][1] = a.y;
						d2[u][0] = c.x;
						d2[u][1] = c.y;
					}
				}
			}
		}
#pragma unroll
		for (int u = 0; u < U; u++) {
#pragma unroll
			for (int j = 0; j < 2; j++) {
				if ((b2[u] >> j) & 1u) {
					const uint64_t oo = o[u] + (j & b2[u]);  // the second slot follows a reported first
					if constexpr (POINTS) {
						Pt rec;
						rec.dim1 = d1[u][j];
						rec.dim2 = d2[u][j];
						if constexpr (HAS_ID)
							rec.id = j ? idv[u].y : idv[u].x;
						static_cast<Pt *>(out)[oo] = rec;
					} else {
						// evict-first: the output streams through L2 once and should not push
						// out tree rows that other queries' records read again
						__stcs(static_cast<uint32_t *>(out) + oo, j ? idv[u].y : idv[u].x);
					}
				}
			}
		}
	}
	__syncwarp();  // the stage is reused by the warp's next batch
}

// THREADS: the CTA size and U the records each warp has in flight (both tuning
// choices; point records keep U = 4).
template <typename T, bool HAS_ID, bool POINTS, int THREADS, int U>
__global__ void __launch_bounds__(THREADS) k_emit(TreeDev<T> t, WorkDev w, void *out, uint64_t capacity)
{
	// a programmatic dependent of the scan (a no-op after any other predecessor)
	asm volatile("griddepcontrol.wait;" ::: "memory");
	__shared__ uint64_t s_total;
	__shared__ EmitStage s_stage[THREADS / 32];
	if (threadIdx.x == 0) {
		uint64_t b = 0;
		for (uint32_t e = 0; e < t.levels; e++)
			b += w.ctl->lvl_cnt[e];
		s_total = b;
	}
	__syncthreads();
	if (w.ctl->total > capacity || (w.ctl->flags & BATCH_FLAG_TASK_OVERFLOW)) {
		if (blockIdx.x == 0 && threadIdx.x == 0 && w.ctl->total > capacity)
			atomicOr(&w.ctl->flags, BATCH_FLAG_OUT_OVERFLOW);
		return;
	}
	const uint64_t total = s_total < w.rec_cap ? s_total : w.rec_cap;
	const uint32_t nro = min(w.ctl->rec_cnt, w.ro_cap);
	const uint32_t lane = lane_id();
	const uint64_t gtid = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
	const uint64_t gwarps = (uint64_t) gridDim.x * blockDim.x / 32, gwarp = gtid / 32;
	// Two batches in flight: the next batch's records are read and its output claimed
	// (an atomic whose result is needed only one batch later) before this batch's
	// results are written.
	const uint64_t stride = gwarps * 32;
	uint64_t wb = gwarp * 32;
	bool v0 = wb + lane < total;
	uint4 m0 = v0 ? w.rec[wb + lane] : make_uint4(0, 0, 0, 0);
	uint64_t ob0 = wb < total ? claim_output(w, m0.y, __popc(m0.z) + __popc(m0.w), v0) : 0;
	guard_claim(w, m0, ob0, capacity);
	while (wb < total) {
		const uint64_t nb = wb + stride;
		const bool v1 = nb + lane < total;
		uint4 m1 = v1 ? w.rec[nb + lane] : make_uint4(0, 0, 0, 0);
		const uint64_t ob1 = nb < total ? claim_output(w, m1.y, __popc(m1.z) + __popc(m1.w), v1) : 0;
		guard_claim(w, m1, ob1, capacity);
		emit_blocks<T, HAS_ID, POINTS, U>(t, m0, ob0, v0, s_stage[threadIdx.x >> 5], out);
		wb = nb;
		v0 = v1;
		m0 = m1;
		ob0 = ob1;
	}
	for (uint64_t wb = gwarp * 32; wb < nro; wb += gwarps * 32) {
		const bool valid = wb + lane < nro;
		uint4 mine = valid ? w.ro[wb + lane] : make_uint4(0, 0, 0, 0);
		const uint64_t ob = claim_output(w, mine.y, __popc(mine.z) + __popc(mine.w), valid);
		guard_claim(w, mine, ob, capacity);
		emit_blocks<T, HAS_ID, POINTS, U>(t, mine, ob, valid, s_stage[threadIdx.x >> 5], out);
	}
}

// Result offsets of a batch in one launch: offsets[q] = the counts of the queries
// before q, offsets[max_q] = ctl->total = all of them.  One CTA walks the counts a
// tile at a time (batches of up to OFFSETS_ONE_CTA queries; larger ones take the
// three-kernel scan).  Launched as a programmatic dependent of the last level.
constexpr uint32_t OFFSETS_ONE_CTA = 4 * SCAN_TILE;

__global__ void __launch_bounds__(SCAN_THREADS) k_offsets(const uint64_t *counts, uint64_t *offsets, uint32_t n,
                                                          BatchCtl *ctl)
{
	asm volatile("griddepcontrol.wait;" ::: "memory");
	__shared__ uint64_t ws[33];
	uint64_t carry = 0;
	for (uint32_t c0 = 0; c0 < n; c0 += SCAN_TILE) {
		const uint32_t base = c0 + threadIdx.x * SCAN_ITEMS;
		uint64_t v[SCAN_ITEMS];
		uint64_t sum = 0;
#pragma unroll
		for (int i = 0; i < SCAN_ITEMS; i++) {
			v[i] = base + i < n ? counts[base + i] : 0;
			sum += v[i];
		}
		uint64_t tot;
		uint64_t ex = block_excl_scan(sum, &tot, ws) + carry;
#pragma unroll
		for (int i = 0; i < SCAN_ITEMS; i++) {
			if (base + i < n)
				offsets[base + i] = ex;
			ex += v[i];
		}
		carry += tot;
	}
	if (threadIdx.x == 0) {
		offsets[n] = carry;
		ctl->total = carry;
	}
}

// Launch configuration of a programmatic dependent of the kernel before it on `s`:
// its CTAs may be scheduled while that kernel drains, and wait (griddepcontrol.wait)
// until it has completed and its writes are visible.
struct DependentLaunch {
	cudaLaunchConfig_t cfg{};
	cudaLaunchAttribute attr[1];
	DependentLaunch(unsigned grid, unsigned threads, cudaStream_t s)
	{
		cfg.gridDim = dim3(grid);
		cfg.blockDim = dim3(threads);
		cfg.dynamicSmemBytes = 0;
		cfg.stream = s;
		attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
		attr[0].val.programmaticStreamSerializationAllowed = 1;
		cfg.attrs = attr;
		cfg.numAttrs = 1;
	}
};

// The batch's result offsets and total (exclusive scan of its counts).
inline void scan_offsets(uint64_t *counts, uint64_t *offsets, uint32_t max_q, uint64_t *scan_tmp, BatchCtl *ctl,
                         cudaStream_t s)
{
	if (max_q <= OFFSETS_ONE_CTA) {
		DependentLaunch l(1, SCAN_THREADS, s);
		PST_CUDA(cudaLaunchKernelEx(&l.cfg, k_offsets, (const uint64_t *) counts, offsets, max_q, ctl));
		return;
	}
	exclusive_scan<uint64_t>(counts, offsets, max_q, scan_tmp, &ctl->total, s);
	PST_CUDA(cudaMemcpyAsync(offsets + max_q, &ctl->total, 8, cudaMemcpyDeviceToDevice, s));
}

// Grid of k_emit: as many CTAs as fit on the device at once (its own occupancy,
// which can differ from the level kernel's), so the grid-stride loop has no tail wave.
template <typename T, bool HAS_ID, bool POINTS, int THREADS, int U>
unsigned emit_grid()
{
	static const int occ = [] {
		int o = 0;
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_emit<T, HAS_ID, POINTS, THREADS, U>, THREADS, 0) !=
		    cudaSuccess) {
			cudaGetLastError();
			o = 1;
		}
		return o > 0 ? o : 1;
	}();
	return (unsigned) (device_info().sms * occ);
}

template <typename T>
void launch_level(const TreeDev<T> &tv, const QDev<T> &qd, const WorkDev &w, uint32_t d, unsigned grid,
                  unsigned threads, cudaStream_t s)
{
	// a programmatic dependent launch: the level's CTAs start as the previous kernel
	// drains (the kernel waits for it before reading anything)
	DependentLaunch l(grid, threads, s);
	cudaLaunchConfig_t &cfg = l.cfg;
	const bool last = d + 1 == tv.levels && tv.last_par;
	switch (threads) {
	case 128:
		PST_CUDA(last ? cudaLaunchKernelEx(&cfg, k_bfs_level<T, true, 128>, tv, qd, w, d)
		              : cudaLaunchKernelEx(&cfg, k_bfs_level<T, false, 128>, tv, qd, w, d));
		break;
	case 512:
		PST_CUDA(last ? cudaLaunchKernelEx(&cfg, k_bfs_level<T, true, 512>, tv, qd, w, d)
		              : cudaLaunchKernelEx(&cfg, k_bfs_level<T, false, 512>, tv, qd, w, d));
		break;
	default:
		PST_CUDA(last ? cudaLaunchKernelEx(&cfg, k_bfs_level<T, true, BFS_THREADS>, tv, qd, w, d)
		              : cudaLaunchKernelEx(&cfg, k_bfs_level<T, false, BFS_THREADS>, tv, qd, w, d));
	}
}

template <typename T>
const void *bfs_kernel_ptr(unsigned threads)
{
	switch (threads) {
	case 128: return reinterpret_cast<const void *>(&k_bfs_level<T, false, 128>);
	case 512: return reinterpret_cast<const void *>(&k_bfs_level<T, false, 512>);
	default: return reinterpret_cast<const void *>(&k_bfs_level<T, false, BFS_THREADS>);
	}
}

// Launches the emit with the batch's CTA size and records in flight.
template <typename T, bool HAS_ID, bool POINTS, int THREADS, int U>
void launch_emit_tu(const TreeDev<T> &tv, const WorkDev &w, void *out, uint64_t capacity, cudaStream_t s)
{
	DependentLaunch l(emit_grid<T, HAS_ID, POINTS, THREADS, U>(), THREADS, s);
	PST_CUDA(cudaLaunchKernelEx(&l.cfg, k_emit<T, HAS_ID, POINTS, THREADS, U>, tv, w, out, capacity));
}

template <typename T, bool HAS_ID, bool POINTS, int THREADS>
void launch_emit_t(const TreeDev<T> &tv, const WorkDev &w, void *out, uint64_t capacity, uint32_t u, cudaStream_t s)
{
	if constexpr (POINTS) {
		(void) u;
		launch_emit_tu<T, HAS_ID, POINTS, THREADS, 4>(tv, w, out, capacity, s);
	} else if (u == 4) {
		launch_emit_tu<T, HAS_ID, POINTS, THREADS, 4>(tv, w, out, capacity, s);
	} else if (u == 16) {
		launch_emit_tu<T, HAS_ID, POINTS, THREADS, 16>(tv, w, out, capacity, s);
	} else {
		launch_emit_tu<T, HAS_ID, POINTS, THREADS, 8>(tv, w, out, capacity, s);
	}
}

template <typename T, bool HAS_ID, bool POINTS>
void launch_emit(const TreeDev<T> &tv, const WorkDev &w, void *out, uint64_t capacity, uint32_t threads, uint32_t u,
                 cudaStream_t s)
{
	switch (threads) {
	case 128: launch_emit_t<T, HAS_ID, POINTS, 128>(tv, w, out, capacity, u, s); break;
	case 512: launch_emit_t<T, HAS_ID, POINTS, 512>(tv, w, out, capacity, u, s); break;
	default: launch_emit_t<T, HAS_ID, POINTS, BFS_THREADS>(tv, w, out, capacity, u, s);
	}
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side.

Batch::~Batch() { release(); }

void Batch::Graph::drop()
{
	if (exec)
		cudaGraphExecDestroy(exec);
	exec = nullptr;
}

void Batch::release()
{
	full_graph.drop();
	top_graph.drop();
	for (void *p : {(void *) q_raw, (void *) kind, min1, max1, min2, (void *) path0, (void *) path1, (void *) seed0,
	                (void *) seed1, (void *) ro, (void *) counts, (void *) cursor, (void *) offsets, (void *) scan_tmp,
	                (void *) ctl, (void *) rec})
		if (p)
			cudaFree(p);
	if (ctl_host)
		cudaFreeHost(ctl_host);
	if (q_stage)
		cudaFreeHost(q_stage);
	q_raw = nullptr;
	ctl_host = nullptr;
	ctl_host_d = nullptr;
	q_stage = nullptr;
	rec = nullptr;
}

static void dmalloc(void **p, size_t bytes)
{
	cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		fail(PST_ERR_NOMEM, "batch workspace allocation of " + std::to_string(bytes) + " B failed");
	}
	check_cuda(e, "cudaMalloc(batch)");
}

void Batch::init(TreeStorage *t, const pst_batch_opts &o)
{
	tree = t;
	max_q = std::max<uint32_t>(o.max_queries, 1);
	use_graph = o.use_graph != 0;
	threads = o.block_threads ? o.block_threads : BFS_THREADS;
	if (threads != 128 && threads != 256 && threads != 512)
		fail(PST_ERR_INVALID, "block_threads must be 0, 128, 256 or 512");
	emit_u = o.emit_records ? o.emit_records : 8;
	if (emit_u != 4 && emit_u != 8 && emit_u != 16)
		fail(PST_ERR_INVALID, "emit_records must be 0, 4, 8 or 16");
	top_q = o.top_pass_queries ? o.top_pass_queries : SMALL_BATCH_Q;
	if (top_q > MAX_TOP_PASS_Q)
		fail(PST_ERR_INVALID, "top_pass_queries must be at most " + std::to_string(MAX_TOP_PASS_Q));
	int occ = 0;
	const void *kfn = nullptr;
	switch (t->dtype) {
	case PST_F32: kfn = bfs_kernel_ptr<float>(threads); cta_pass_budget<float>(); break;
	case PST_F64: kfn = bfs_kernel_ptr<double>(threads); cta_pass_budget<double>(); break;
	case PST_I32: kfn = bfs_kernel_ptr<int32_t>(threads); cta_pass_budget<int32_t>(); break;
	}
	PST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, threads, 0));
	blocks_per_sm = o.blocks_per_sm ? std::min<uint32_t>(o.blocks_per_sm, (uint32_t) std::max(occ, 1))
	                                : (uint32_t) std::max(occ, 1);
	grid = (uint32_t) device_info().sms * blocks_per_sm;
	const size_t vs = value_size(t->dtype);
	path_cap = 2 * max_q;
	ro_cap = 2 * max_q * 32;
	dmalloc((void **) &q_raw, (size_t) max_q * sizeof(pst_query));
	dmalloc((void **) &kind, (size_t) max_q * 4);
	dmalloc(&min1, (size_t) max_q * vs);
	dmalloc(&max1, (size_t) max_q * vs);
	dmalloc(&min2, (size_t) max_q * vs);
	dmalloc((void **) &path0, (size_t) path_cap * sizeof(uint4));
	dmalloc((void **) &path1, (size_t) path_cap * sizeof(uint4));
	dmalloc((void **) &seed0, (size_t) path_cap * sizeof(uint4));
	dmalloc((void **) &seed1, (size_t) path_cap * sizeof(uint4));
	dmalloc((void **) &ro, (size_t) ro_cap * sizeof(uint4));
	dmalloc((void **) &counts, (size_t) max_q * 8);
	dmalloc((void **) &cursor, (size_t) max_q * 8);
	dmalloc((void **) &offsets, ((size_t) max_q + 1) * 8);
	dmalloc((void **) &scan_tmp, scan_tmp_elems(max_q) * 8);
	dmalloc((void **) &ctl, sizeof(BatchCtl));
	PST_CUDA(cudaMallocHost((void **) &ctl_host, sizeof(BatchCtl)));
	PST_CUDA(cudaMallocHost((void **) &q_stage, (size_t) max_q * sizeof(pst_query)));
	memset(ctl_host, 0, sizeof(BatchCtl));
	PST_CUDA(cudaHostGetDevicePointer((void **) &ctl_host_d, ctl_host, 0));
	const uint64_t want = o.task_capacity ? o.task_capacity : std::max<uint64_t>(1ull << 16, (uint64_t) max_q * 64);
	grow_tasks(want, 0);
	PST_CUDA(cudaStreamSynchronize(0));
}

void Batch::grow_tasks(uint64_t cap, cudaStream_t s)
{
	// Stream-ordered on `s` (the stream of every pass that used the old frontier), so
	// a growth does not wait for work on the device's other streams.
	if (rec)
		PST_CUDA(cudaFreeAsync(rec, s));
	rec = nullptr;
	const size_t bytes = std::max<size_t>(cap * sizeof(uint4), 16);
	cudaError_t e = cudaMallocAsync((void **) &rec, bytes, s);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		task_cap = 0;
		fail(PST_ERR_NOMEM, "frontier allocation of " + std::to_string(bytes) + " B failed");
	}
	check_cuda(e, "cudaMallocAsync(frontier)");
	task_cap = cap;
	// the captured passes hold the old frontier's address
	full_graph.drop();
	top_graph.drop();
}

#define PST_WORKDEV                                                                                                   \
	WorkDev w{rec, task_cap, path0, path1, seed0, seed1, path_cap, ro, ro_cap, counts, cursor, offsets, ctl}

template <typename T>
void Batch::enqueue_count(cudaStream_t s)
{
	TreeDev<T> tv = tree->view<T>();
	QDev<T> qd{kind, static_cast<const T *>(min1), static_cast<const T *>(max1), static_cast<const T *>(min2)};
	PST_WORKDEV;
	k_load_ctl<<<1, 256, 0, s>>>(ctl_host_d, ctl);
	const unsigned ug = (unsigned) std::min<uint64_t>((max_q + 255) / 256, (uint64_t) device_info().sms * 4);
	const QOut<T> qo{kind, static_cast<T *>(min1), static_cast<T *>(max1), static_cast<T *>(min2)};
	k_prepare_queries<T><<<ug, 256, 0, s>>>(q_raw, ctl, qo, path0, counts, cursor, max_q);
	for (uint32_t d = 0; d < tv.levels; d++)
		launch_level<T>(tv, qd, w, d, grid, threads, s);
	scan_offsets(counts, offsets, max_q, scan_tmp, ctl, s);
	PST_CUDA(cudaGetLastError());
}

template <typename T>
void Batch::enqueue_count_top(cudaStream_t s)
{
	TreeDev<T> tv = tree->view<T>();
	QDev<T> qd{kind, static_cast<const T *>(min1), static_cast<const T *>(max1), static_cast<const T *>(min2)};
	PST_WORKDEV;
	// one kernel: the control block read from its pinned host copy, the queries
	// unpacked and the whole top pass
	const QOut<T> qo{kind, static_cast<T *>(min1), static_cast<T *>(max1), static_cast<T *>(min2)};
	launch_cta_pass<T>(tv, qd, w, max_q, 2 * std::min(top_q, max_q), q_raw, qo, ctl_host_d, s);
	PST_CUDA(cudaGetLastError());
}

template <typename T>
void Batch::enqueue_count_rest(uint32_t from, cudaStream_t s)
{
	TreeDev<T> tv = tree->view<T>();
	QDev<T> qd{kind, static_cast<const T *>(min1), static_cast<const T *>(max1), static_cast<const T *>(min2)};
	PST_WORKDEV;
	for (uint32_t d = from; d < tv.levels; d++)
		launch_level<T>(tv, qd, w, d, grid, threads, s);
	scan_offsets(counts, offsets, max_q, scan_tmp, ctl, s);
	PST_CUDA(cudaGetLastError());
}

template <typename T, bool HAS_ID, bool POINTS>
void Batch::enqueue_emit_t(void *out, uint64_t capacity, cudaStream_t s)
{
	TreeDev<T> tv = tree->view<T>();
	PST_WORKDEV;
	launch_emit<T, HAS_ID, POINTS>(tv, w, out, capacity, threads, emit_u, s);
	PST_CUDA(cudaGetLastError());
}

template <typename T>
void Batch::enqueue_emit_v(pst_ret ret, void *out, uint64_t capacity, cudaStream_t s)
{
	const bool has_id = tree->idtype == PST_ID_U32;
	if (ret == PST_RET_IDS) {
		if (!has_id)
			fail(PST_ERR_UNSUPPORTED, "an id-less tree can only return points");
		enqueue_emit_t<T, true, false>(out, capacity, s);
	} else if (has_id) {
		enqueue_emit_t<T, true, true>(out, capacity, s);
	} else {
		enqueue_emit_t<T, false, true>(out, capacity, s);
	}
}

void Batch::enqueue_counting(cudaStream_t s)
{
	switch (tree->dtype) {
	case PST_F32: enqueue_count<float>(s); break;
	case PST_F64: enqueue_count<double>(s); break;
	case PST_I32: enqueue_count<int32_t>(s); break;
	}
}

void Batch::enqueue_counting_top(cudaStream_t s)
{
	switch (tree->dtype) {
	case PST_F32: enqueue_count_top<float>(s); break;
	case PST_F64: enqueue_count_top<double>(s); break;
	case PST_I32: enqueue_count_top<int32_t>(s); break;
	}
}

void Batch::enqueue_emit(pst_ret ret, void *out, uint64_t capacity, cudaStream_t s)
{
	switch (tree->dtype) {
	case PST_F32: enqueue_emit_v<float>(ret, out, capacity, s); break;
	case PST_F64: enqueue_emit_v<double>(ret, out, capacity, s); break;
	case PST_I32: enqueue_emit_v<int32_t>(ret, out, capacity, s); break;
	}
}

void Batch::launch_graph(Graph &g, void (Batch::*enqueue)(cudaStream_t), cudaStream_t s)
{
	if (!use_graph) {
		(this->*enqueue)(s);
		return;
	}
	if (!g.exec || g.stream != s) {
		g.drop();
		cudaStream_t cs;
		PST_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
		cudaGraph_t gr;
		PST_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
		try {
			(this->*enqueue)(cs);
		} catch (...) {
			cudaStreamEndCapture(cs, &gr);
			cudaStreamDestroy(cs);
			throw;
		}
		PST_CUDA(cudaStreamEndCapture(cs, &gr));
		PST_CUDA(cudaGraphInstantiate(&g.exec, gr, 0));
		cudaGraphDestroy(gr);
		cudaStreamDestroy(cs);
		g.stream = s;
	}
	PST_CUDA(cudaGraphLaunch(g.exec, s));
}

void Batch::launch_count(cudaStream_t s) { launch_graph(full_graph, &Batch::enqueue_counting, s); }

void Batch::launch_count_top(cudaStream_t s)
{
	if (ctl_host->nq > top_q)
		fail(PST_ERR_INTERNAL, "top pass on a batch of more than " + std::to_string(top_q) + " queries");
	launch_graph(top_graph, &Batch::enqueue_counting_top, s);
}

void Batch::launch_count_rest(uint32_t from, cudaStream_t s)
{
	switch (tree->dtype) {
	case PST_F32: enqueue_count_rest<float>(from, s); break;
	case PST_F64: enqueue_count_rest<double>(from, s); break;
	case PST_I32: enqueue_count_rest<int32_t>(from, s); break;
	}
}

void Batch::stage_queries(const pst_query *q, uint32_t nq, bool on_device, cudaStream_t s)
{
	if (nq > max_q)
		fail(PST_ERR_INVALID, "batch of " + std::to_string(nq) + " queries exceeds max_queries " +
		                          std::to_string(max_q));
	if (nq && !q)
		fail(PST_ERR_INVALID, "null query array");
	// the pinned control block and query staging may still feed an earlier pass
	PST_CUDA(cudaStreamSynchronize(s));
	ctl_host->nq = nq;
	if (nq) {
		if (on_device) {
			PST_CUDA(cudaMemcpyAsync(q_raw, q, (size_t) nq * sizeof(pst_query), cudaMemcpyDeviceToDevice, s));
		} else {
			memcpy(q_stage, q, (size_t) nq * sizeof(pst_query));
			PST_CUDA(cudaMemcpyAsync(q_raw, q_stage, (size_t) nq * sizeof(pst_query), cudaMemcpyHostToDevice, s));
		}
	}
}

pst_status Batch::read_ctl(cudaStream_t s, uint64_t *total)
{
	BatchCtl h;
	PST_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaStreamSynchronize(s));
	last = h;
	if (total)
		*total = h.total;
	if (h.flags & BATCH_FLAG_BAD_QUERY)
		return PST_ERR_INVALID;
	if (h.flags & (BATCH_FLAG_TASK_OVERFLOW | BATCH_FLAG_INTERNAL))
		return PST_ERR_INTERNAL;
	if (h.flags & BATCH_FLAG_OUT_OVERFLOW)
		return PST_ERR_CAPACITY;
	return PST_OK;
}

// Count pass with the host waiting for it.
void Batch::count_sync(cudaStream_t s, uint64_t *total)
{
	if (ctl_host->nq <= top_q)
		count_small_sync(s, total);
	else
		count_full_sync(s, total);
}

// Reads the control block after a pass; true when it is complete, false when the
// frontier overflowed (and has been grown for another attempt).
static bool settle(Batch &b, const BatchCtl &h, int attempt, cudaStream_t s, uint64_t *total)
{
	b.last = h;
	if (h.flags & BATCH_FLAG_BAD_QUERY)
		fail(PST_ERR_INVALID, "query kind must be PST_Q_THREE, PST_Q_LEFT or PST_Q_RIGHT");
	if (h.flags & BATCH_FLAG_INTERNAL)
		fail(PST_ERR_INTERNAL, "search consistency check failed");
	if (!(h.flags & BATCH_FLAG_TASK_OVERFLOW)) {
		*total = h.total;
		return true;
	}
	if (attempt > 8)
		fail(PST_ERR_INTERNAL, "frontier did not fit after growth");
	b.grow_tasks(std::max<uint64_t>(h.need_tasks + h.need_tasks / 4, b.task_cap * 2), s);
	return false;
}

// The whole pass, with automatic growth of the frontier buffer.
void Batch::count_full_sync(cudaStream_t s, uint64_t *total)
{
	for (int attempt = 0;; attempt++) {
		launch_count(s);
		BatchCtl h;
		PST_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
		PST_CUDA(cudaStreamSynchronize(s));
		if (settle(*this, h, attempt, s, total))
			return;
	}
}

// A small batch: the one-CTA top pass, then, if it stopped above the bottom, the
// per-level kernels for the rest and the scan; with automatic growth of the
// frontier buffer as in count_full_sync.
void Batch::count_small_sync(cudaStream_t s, uint64_t *total)
{
	for (int attempt = 0;; attempt++) {
		launch_count_top(s);
		BatchCtl h;
		PST_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
		PST_CUDA(cudaStreamSynchronize(s));
		if (!(h.flags & (BATCH_FLAG_BAD_QUERY | BATCH_FLAG_INTERNAL | BATCH_FLAG_TASK_OVERFLOW)) &&
		    h.cta_levels < tree->levels) {
			launch_count_rest(h.cta_levels, s);
			PST_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
			PST_CUDA(cudaStreamSynchronize(s));
		}
		if (settle(*this, h, attempt, s, total))
			return;
	}
}

uint64_t Batch::record_size(pst_ret ret) const
{
	return ret == PST_RET_IDS ? 4 : point_size(tree->dtype, tree->idtype);
}

// ---------------------------------------------------------------------------
// Single query with no allocation at all (pst_search_noalloc).
//
// For callers that cannot allocate device memory during a search: code whose
// device memory is all owned by its own allocator (so a cudaMalloc here would fail
// or compete with it), and latency-critical loops that cannot take the implicit
// device-wide synchronisation of cudaMalloc/cudaFree.  The search's working memory
// (control block, the query, its boundary paths and its frontier) lives in the
// file-scope array below, which every GPU that loads this library holds until the
// process exits.

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(8) << 20;  // 8 MiB per device
constexpr uint32_t NOALLOC_MAX_LEVELS = 22;                  // trees of up to 2^22 - 1 points

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Sub-buffers of the scratch array, 256-byte aligned, in bytes.
constexpr size_t NA_CTL = 0;
constexpr size_t NA_QRAW = 1024;
constexpr size_t NA_KIND = NA_QRAW + 256;
constexpr size_t NA_MIN1 = NA_KIND + 256;
constexpr size_t NA_MAX1 = NA_MIN1 + 256;
constexpr size_t NA_MIN2 = NA_MAX1 + 256;
constexpr size_t NA_PATH0 = NA_MIN2 + 256;
constexpr size_t NA_PATH1 = NA_PATH0 + 256;
constexpr size_t NA_SEED0 = NA_PATH1 + 256;
constexpr size_t NA_SEED1 = NA_SEED0 + 256;
constexpr uint32_t NA_RO_CAP = 2 * 32;  // two boundary results per level
constexpr size_t NA_RO = NA_SEED1 + 256;
constexpr size_t NA_COUNTS = NA_RO + NA_RO_CAP * sizeof(uint4);
constexpr size_t NA_CURSOR = NA_COUNTS + 256;
constexpr size_t NA_OFFSETS = NA_CURSOR + 256;
constexpr size_t NA_SCAN = NA_OFFSETS + 256;
constexpr size_t NA_RECS = NA_SCAN + 256;
// alive records (16 B each) take the rest
constexpr uint64_t NA_REC_CAP = (NOALLOC_SCRATCH_BYTES - NA_RECS) / sizeof(uint4) / 64 * 64;
static_assert(sizeof(BatchCtl) <= NA_QRAW, "control block");
static_assert(NA_RECS + NA_REC_CAP * sizeof(uint4) <= NOALLOC_SCRATCH_BYTES, "scratch layout");
// One query has at most one alive record per 64-slot block of every level, plus the
// records of report-above subtrees that still share a block with another subtree:
// a seed's subtree shares blocks for its first six levels and a query leaves at
// most two seeds per level, so at most 12 more per level: fewer than
// 2^L/32 + 14L + 64 records for a tree of L levels.
static_assert((1ull << NOALLOC_MAX_LEVELS) / 32 + 14 * NOALLOC_MAX_LEVELS + 64 <= NA_REC_CAP, "frontier bound");

std::mutex g_noalloc_mu;

// The scratch array's device address per device, with the id of the context it was
// looked up in.  cudaDeviceReset ends that context (and the array with it); the next
// call on the device, in the new context, looks the address up again.
struct NoallocSlot {
	unsigned long long ctx = 0;
	unsigned char *ptr = nullptr;
};
NoallocSlot g_noalloc_slot[64];

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current context, made current first for device
// `dev` when the thread has none yet (the library does not link the driver library
// itself: the two driver calls come from the runtime's entry points).
unsigned long long current_context_id(int dev)
{
	static CtxGetCurrentFn get_cur = nullptr;
	static CtxGetIdFn get_id = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			get_cur = reinterpret_cast<CtxGetCurrentFn>(p);
		p = nullptr;
		if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			get_id = reinterpret_cast<CtxGetIdFn>(p);
		cudaGetLastError();
	});
	if (!get_cur || !get_id)
		fail(PST_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId are unavailable");
	CUcontext c = nullptr;
	if (get_cur(&c) == CUDA_SUCCESS && !c) {
		// a thread that has made no other CUDA call: cudaSetDevice makes the device's
		// primary context current on it
		check_cuda(cudaSetDevice(dev), "cudaSetDevice");
		get_cur(&c);
	}
	unsigned long long id = 0;
	if (!c || get_id(c, &id) != CUDA_SUCCESS)
		fail(PST_ERR_CUDA, "no current CUDA context");
	return id;
}

// Device address of the scratch array for device `dev`, which must be current
// (the host-side name of a __device__ array is only a stand-in for it): looked up
// once per device and context.
unsigned char *noalloc_scratch(int dev)
{
	if (dev < 0 || dev >= 64)
		fail(PST_ERR_CUDA, "device index out of range");
	const unsigned long long ctx = current_context_id(dev);
	NoallocSlot &slot = g_noalloc_slot[dev];
	if (!slot.ptr || slot.ctx != ctx) {
		void *p = nullptr;
		check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
		slot.ptr = static_cast<unsigned char *>(p);
		slot.ctx = ctx;
	}
	return slot.ptr;
}

template <typename T>
uint64_t noalloc_run(TreeStorage &t, const pst_query &q, pst_ret ret, void *out, uint64_t capacity, cudaStream_t s,
                     unsigned char *base)
{
	BatchCtl *ctl = reinterpret_cast<BatchCtl *>(base + NA_CTL);
	pst_query *qraw = reinterpret_cast<pst_query *>(base + NA_QRAW);
	uint32_t *kind = reinterpret_cast<uint32_t *>(base + NA_KIND);
	T *min1 = reinterpret_cast<T *>(base + NA_MIN1);
	T *max1 = reinterpret_cast<T *>(base + NA_MAX1);
	T *min2 = reinterpret_cast<T *>(base + NA_MIN2);
	uint4 *path0 = reinterpret_cast<uint4 *>(base + NA_PATH0);
	uint4 *path1 = reinterpret_cast<uint4 *>(base + NA_PATH1);
	uint4 *seed0 = reinterpret_cast<uint4 *>(base + NA_SEED0);
	uint4 *seed1 = reinterpret_cast<uint4 *>(base + NA_SEED1);
	uint4 *ro = reinterpret_cast<uint4 *>(base + NA_RO);
	uint64_t *counts = reinterpret_cast<uint64_t *>(base + NA_COUNTS);
	uint64_t *cursor = reinterpret_cast<uint64_t *>(base + NA_CURSOR);
	uint64_t *offsets = reinterpret_cast<uint64_t *>(base + NA_OFFSETS);
	uint64_t *scan = reinterpret_cast<uint64_t *>(base + NA_SCAN);
	uint4 *rec = reinterpret_cast<uint4 *>(base + NA_RECS);

	// The array keeps the previous call's contents: the control block starts over
	// (with nq = 1) here, and the top pass zeroes the query's count and output cursor.
	BatchCtl h{};
	h.nq = 1;
	PST_CUDA(cudaMemcpyAsync(ctl, &h, sizeof(BatchCtl), cudaMemcpyHostToDevice, s));
	PST_CUDA(cudaMemcpyAsync(qraw, &q, sizeof(pst_query), cudaMemcpyHostToDevice, s));

	int occ = 0;
	PST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bfs_kernel_ptr<T>(BFS_THREADS), BFS_THREADS, 0));
	const unsigned grid = (unsigned) device_info().sms * (unsigned) std::max(occ, 1);
	TreeDev<T> tv = t.view<T>();
	QDev<T> qd{kind, min1, max1, min2};
	WorkDev w{rec, NA_REC_CAP, path0, path1, seed0, seed1, 2u, ro, NA_RO_CAP, counts, cursor, offsets, ctl};
	// the one-CTA top pass (which unpacks the query and zeroes its count and output
	// cursor), then the per-level kernels for whatever it left
	launch_cta_pass<T>(tv, qd, w, 1u, 2u, qraw, QOut<T>{kind, min1, max1, min2}, ctl, s);
	PST_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaStreamSynchronize(s));
	if (!(h.flags & (BATCH_FLAG_BAD_QUERY | BATCH_FLAG_INTERNAL | BATCH_FLAG_TASK_OVERFLOW)) &&
	    h.cta_levels < tv.levels) {
		for (uint32_t d = h.cta_levels; d < tv.levels; d++)
			launch_level<T>(tv, qd, w, d, grid, BFS_THREADS, s);
		scan_offsets(counts, offsets, 1, scan, ctl, s);
		PST_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
		PST_CUDA(cudaStreamSynchronize(s));
	}
	if (h.flags & BATCH_FLAG_BAD_QUERY)
		fail(PST_ERR_INVALID, "query kind must be PST_Q_THREE, PST_Q_LEFT or PST_Q_RIGHT");
	if (h.flags & (BATCH_FLAG_TASK_OVERFLOW | BATCH_FLAG_INTERNAL))
		fail(PST_ERR_INTERNAL, "no-alloc search: frontier consistency check failed");
	if (h.total == 0 || h.total > capacity)
		return h.total;
	const bool has_id = t.idtype == PST_ID_U32;
	if (ret == PST_RET_IDS)
		launch_emit<T, true, false>(tv, w, out, capacity, BFS_THREADS, 8, s);
	else if (has_id)
		launch_emit<T, true, true>(tv, w, out, capacity, BFS_THREADS, 4, s);
	else
		launch_emit<T, false, true>(tv, w, out, capacity, BFS_THREADS, 4, s);
	PST_CUDA(cudaGetLastError());
	PST_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaStreamSynchronize(s));
	if (h.flags & (BATCH_FLAG_OUT_OVERFLOW | BATCH_FLAG_INTERNAL))
		fail(PST_ERR_INTERNAL, "no-alloc search: emit consistency check failed");
	return h.total;
}

}  // namespace

uint64_t search_noalloc(TreeStorage &t, const pst_query &q, pst_ret ret, void *out, uint64_t capacity, cudaStream_t s)
{
	if (t.levels > NOALLOC_MAX_LEVELS)
		fail(PST_ERR_CAPACITY, "pst_search_noalloc handles trees of at most " +
		                           std::to_string((1ull << NOALLOC_MAX_LEVELS) - 1) + " points (" +
		                           std::to_string(NOALLOC_SCRATCH_BYTES >> 20) + " MiB static scratch); this tree has " +
		                           std::to_string(t.n));
	int dev = 0;
	PST_CUDA(cudaGetDevice(&dev));
	if (t.device != dev)
		fail(PST_ERR_INVALID, "the tree lives on device " + std::to_string(t.device) + " but device " +
		                          std::to_string(dev) + " is current");
	// Every call on a device shares the one array, so two calls whose GPU work
	// overlapped would race on it; within this process the lock, held until the
	// call's work has completed, keeps calls from overlapping.
	std::lock_guard<std::mutex> lk(g_noalloc_mu);
	unsigned char *base = noalloc_scratch(dev);
	try {
		switch (t.dtype) {
		case PST_F32: return noalloc_run<float>(t, q, ret, out, capacity, s, base);
		case PST_F64: return noalloc_run<double>(t, q, ret, out, capacity, s, base);
		case PST_I32: return noalloc_run<int32_t>(t, q, ret, out, capacity, s, base);
		}
	} catch (...) {
		// kernels enqueued before the failure may still be using the array: let them
		// finish before the lock is released and another call rewrites it
		cudaStreamSynchronize(s);
		cudaGetLastError();
		throw;
	}
	fail(PST_ERR_INVALID, "bad dtype");
}

}  // namespace pst
