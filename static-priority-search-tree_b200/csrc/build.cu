// Construction of the static priority search tree on the GPU.
//
// The tree is the one the reference's StaticPSTCPUIter builds, node for node
// (pst/static-pst-cpu-iter.tpp:18-177, pst/static-pst-cpu-iter-populate-tree.tpp:11-114,
// constructNode at pst/static-pst-cpu-iter.tpp:491-598):
//   - a node of c points holds the point that is largest in the dim2 order
//     (value, then id, then input index: helpers/point-struct.h:62-92, :154-188);
//   - its median is the dim1 value of the floor(c/2)-th of the remaining points in
//     dim1 order, and those floor(c/2) points form the left subtree;
//   - the rest form the right subtree.
// The reference finds each node's point with a binary search, then shifts and
// partitions index arrays one node at a time (pst/static-pst-gpu.tu:678-806; one
// thread per node, one block, dynamic parallelism).  This build works level by level
// instead:
//   1. one radix sort ranks the points in dim1 order and one in dim2 order;
//   2. for the wide top levels, a streaming segmented arg-max over the dim1-ordered
//      dim2 ranks picks every node's point of the level at once, and a per-node
//      kernel places the median.  Points already taken by ancestors are zeroed
//      and so drop out of later maxima;
//   3. once every node of a level holds at most ST_CAP points, one CTA per node
//      builds the whole remaining subtree in shared memory.
#include <algorithm>
#include <vector>

#include "scan_sort.cuh"
#include "tree.cuh"

namespace pst {

size_t value_size(pst_dtype dt) { return dt == PST_F64 ? 8 : 4; }

size_t point_size(pst_dtype dt, pst_idtype it)
{
	if (dt != PST_F32 && dt != PST_F64 && dt != PST_I32)
		return 0;
	if (it == PST_ID_NONE)
		return 2 * value_size(dt);
	if (it == PST_ID_U32)
		return dt == PST_F64 ? 24 : 12;
	return 0;
}

namespace {

constexpr size_t ALIGN = 256;
inline size_t align_up(size_t v) { return (v + ALIGN - 1) / ALIGN * ALIGN; }

struct TreeLayout {
	size_t off_dim1, off_dim2, off_med, off_id, off_occ, total;
};

TreeLayout tree_layout(pst_dtype dt, pst_idtype it, uint64_t n)
{
	TreeLayout L{};
	if (n == 0)
		return L;
	const uint32_t D = tree_levels(n);
	const uint64_t S = 1ull << D;
	const size_t vs = value_size(dt);
	size_t o = 0;
	L.off_dim1 = o;
	o = align_up(o + S * vs);
	L.off_dim2 = o;
	o = align_up(o + S * vs);
	L.off_med = o;
	o = align_up(o + (S / 2) * vs);
	L.off_id = o;
	if (it == PST_ID_U32)
		o = align_up(o + S * 4);
	L.off_occ = o;
	o = align_up(o + std::max<uint64_t>(S / 32, 1) * 4);
	L.total = o;
	return L;
}

// Subtree builder capacity: nodes of at most ST_CAP points are finished by one CTA.
constexpr uint32_t ST_CAP = 2048;
constexpr int ST_THREADS = 256;
// Arg-max tile: every segment of a level before the subtree level spans at least
// ST_CAP >= AM_TILE positions, so a tile meets at most two segments.
constexpr int AM_THREADS = 256;
constexpr int AM_ITEMS = 8;
constexpr uint32_t AM_TILE = AM_THREADS * AM_ITEMS;
static_assert(ST_CAP >= AM_TILE, "tile/segment invariant");

// First level whose largest node holds at most ST_CAP points.  Counts within a
// level take at most two consecutive values (m, m+1).
uint32_t subtree_level(uint64_t n)
{
	uint64_t hi = n;
	uint32_t d = 0;
	while (hi > ST_CAP) {
		hi = hi / 2;  // largest child of the largest node
		d++;
	}
	return d;
}

template <typename T, bool HAS_ID>
struct BuildCtx {
	const Point<T, HAS_ID> *pts;
	const uint32_t *P;       // tiebreak rank -> input index (null: identity)
	const uint32_t *S1;      // dim1-sorted position -> tiebreak rank
	uint32_t *r2p1;          // dim1-sorted position -> dim2 rank + 1 (0 once taken)
	const uint32_t *pos_of_rank2;
	T *dim1;
	T *dim2;
	T *med;
	uint32_t *id;
	uint32_t *occ;
	uint32_t *top_pos;       // heap position -> dim1-sorted position of its point (levels < L0)
	uint32_t *err;
	uint64_t n;
	uint32_t D;

	__device__ __forceinline__ Point<T, HAS_ID> point_at(uint32_t pos) const
	{
		const uint32_t tb = S1[pos];
		return pts[P ? P[tb] : tb];
	}

	__device__ __forceinline__ void write_node(uint32_t h, const Point<T, HAS_ID> &p) const
	{
		dim1[h] = p.dim1;
		dim2[h] = p.dim2;
		if constexpr (HAS_ID)
			id[h] = p.id;
	}
};

// ---------------------------------------------------------------------------
// Preparation kernels.

template <typename T, bool HAS_ID>
__global__ void k_ids_monotone(const Point<T, HAS_ID> *pts, uint64_t n, uint32_t *flag)
{
	if constexpr (HAS_ID) {
		for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n;
		     i += (uint64_t) gridDim.x * blockDim.x)
			if (pts[i].id > pts[i + 1].id) {
				atomicOr(flag, 1u);
				return;
			}
	}
}

template <typename T, bool HAS_ID>
__global__ void k_id_keys(const Point<T, HAS_ID> *pts, uint64_t n, uint32_t *keys)
{
	if constexpr (HAS_ID) {
		for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t) gridDim.x * blockDim.x)
			keys[i] = pts[i].id;
	}
}

// Keys of both dimensions in tiebreak-rank order r (input index P[r]).
template <typename T, bool HAS_ID>
__global__ void k_value_keys(const Point<T, HAS_ID> *pts, const uint32_t *P, uint64_t n, typename KeyOf<T>::K *k1,
                             typename KeyOf<T>::K *k2)
{
	for (uint64_t r = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t) gridDim.x * blockDim.x) {
		const Point<T, HAS_ID> p = pts[P ? P[r] : r];
		k1[r] = KeyOf<T>::key(p.dim1);
		k2[r] = KeyOf<T>::key(p.dim2);
	}
}

__global__ void k_iota(uint32_t *v, uint64_t n)
{
	for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t) gridDim.x * blockDim.x)
		v[i] = (uint32_t) i;
}

__global__ void k_rank_scatter(const uint32_t *S2, uint64_t n, uint32_t *rank2_of_tb)
{
	for (uint64_t j = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t) gridDim.x * blockDim.x)
		rank2_of_tb[S2[j]] = (uint32_t) j;
}

__global__ void k_sorted_ranks(const uint32_t *S1, const uint32_t *rank2_of_tb, uint64_t n, uint32_t *r2p1,
                               uint32_t *pos_of_rank2)
{
	for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t) gridDim.x * blockDim.x) {
		const uint32_t rk = rank2_of_tb[S1[i]];
		r2p1[i] = rk + 1;
		pos_of_rank2[rk] = (uint32_t) i;
	}
}

// ---------------------------------------------------------------------------
// Wide levels.

// best[s] = max r2p1 over positions [B[s], B[s+1]).  Each CTA walks a contiguous
// run of tiles and keeps the open segment's running maximum, so a segment costs
// one global atomic per CTA that touches it.
__global__ void __launch_bounds__(AM_THREADS) k_level_argmax(const uint32_t *__restrict__ r2p1, uint64_t n,
                                                             const uint32_t *__restrict__ B, uint32_t nseg,
                                                             uint32_t *best, uint64_t tiles_per_cta)
{
	__shared__ uint32_t s_red[2][AM_THREADS / 32];
	__shared__ uint32_t s_seg;
	const uint64_t num_tiles = (n + AM_TILE - 1) / AM_TILE;
	const uint64_t tb = (uint64_t) blockIdx.x * tiles_per_cta;
	const uint64_t te = min(tb + tiles_per_cta, num_tiles);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	uint32_t run_seg = 0xFFFFFFFFu, run_max = 0;  // thread 0 only
	for (uint64_t tile = tb; tile < te; tile++) {
		const uint64_t t0 = tile * AM_TILE;
		if (threadIdx.x == 0) {
			uint32_t lo = 0, hi = nseg;  // largest s in [0, nseg) with B[s] <= t0
			while (hi - lo > 1) {
				uint32_t mid = (lo + hi) / 2;
				if (B[mid] <= t0)
					lo = mid;
				else
					hi = mid;
			}
			s_seg = lo;
		}
		__syncthreads();
		const uint32_t sa = s_seg;
		const uint64_t bnd = sa + 1 < nseg ? B[sa + 1] : n;
		uint32_t ma = 0, mb = 0;
		const uint64_t base = t0 + (uint64_t) threadIdx.x * AM_ITEMS;
		uint32_t v[AM_ITEMS];
		if (base + AM_ITEMS <= n && (reinterpret_cast<uintptr_t>(r2p1 + base) & 15) == 0) {
			const uint4 a = *reinterpret_cast<const uint4 *>(r2p1 + base);
			const uint4 b = *reinterpret_cast<const uint4 *>(r2p1 + base + 4);
			v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
			v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
		} else {
#pragma unroll
			for (int e = 0; e < AM_ITEMS; e++)
				v[e] = base + e < n ? r2p1[base + e] : 0u;
		}
#pragma unroll
		for (int e = 0; e < AM_ITEMS; e++) {
			if (base + e < bnd)
				ma = max(ma, v[e]);
			else
				mb = max(mb, v[e]);
		}
		ma = __reduce_max_sync(0xFFFFFFFFu, ma);
		mb = __reduce_max_sync(0xFFFFFFFFu, mb);
		if (lane == 0) {
			s_red[0][warp] = ma;
			s_red[1][warp] = mb;
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			uint32_t MA = 0, MB = 0;
			for (int w = 0; w < AM_THREADS / 32; w++) {
				MA = max(MA, s_red[0][w]);
				MB = max(MB, s_red[1][w]);
			}
			if (run_seg == sa) {
				run_max = max(run_max, MA);
			} else {
				if (run_seg != 0xFFFFFFFFu)
					atomicMax(&best[run_seg], run_max);
				run_seg = sa;
				run_max = MA;
			}
			if (bnd < (t0 + AM_TILE < n ? t0 + AM_TILE : n)) {  // the tile reaches segment sa + 1
				atomicMax(&best[run_seg], run_max);
				run_seg = sa + 1;
				run_max = MB;
			}
		}
		__syncthreads();
	}
	if (threadIdx.x == 0 && run_seg != 0xFFFFFFFFu)
		atomicMax(&best[run_seg], run_max);
}

// One thread per node of level d: take the arg-max point, place the median, write
// the node and the next level's segment bounds.  Bounds are dim1-sorted positions
// that still include points taken by ancestors; those (at most d of them inside a
// segment, each the point of one ancestor) are skipped when counting to the median.
template <typename T, bool HAS_ID>
__global__ void k_level_nodes(BuildCtx<T, HAS_ID> c, uint32_t d, const uint32_t *__restrict__ B,
                              uint32_t *__restrict__ Bn, const uint32_t *__restrict__ best)
{
	const uint32_t nseg = 1u << d;
	const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nseg)
		return;
	const uint32_t h = nseg + j;
	const uint64_t cnt = node_count(c.n, d, j);
	const uint32_t lo = B[j], hi = B[j + 1];
	const uint32_t bj = best[j];
	if (bj == 0 || cnt < 2) {
		atomicOr(c.err, 1u);
		return;
	}
	const uint32_t tp = c.pos_of_rank2[bj - 1];
	c.r2p1[tp] = 0;
	c.top_pos[h] = tp;
	uint32_t rem[33];
	uint32_t nr = 0;
	rem[nr++] = tp;
	for (uint32_t a = h >> 1; a >= 1; a >>= 1) {
		const uint32_t ta = c.top_pos[a];
		if (ta >= lo && ta < hi)
			rem[nr++] = ta;
	}
	for (uint32_t i = 1; i < nr; i++) {  // insertion sort, nr <= d + 1
		const uint32_t x = rem[i];
		uint32_t k = i;
		while (k > 0 && rem[k - 1] > x) {
			rem[k] = rem[k - 1];
			k--;
		}
		rem[k] = x;
	}
	uint32_t pos = lo + (uint32_t) (cnt / 2) - 1;
	for (uint32_t i = 0; i < nr; i++)
		if (rem[i] <= pos)
			pos++;
	if (pos >= hi) {
		atomicOr(c.err, 4u);
		return;
	}
	Bn[2 * j] = lo;
	Bn[2 * j + 1] = pos + 1;
	if (j == nseg - 1)
		Bn[2 * nseg] = hi;
	c.write_node(h, c.point_at(tp));
	c.med[h] = c.point_at(pos).dim1;
	atomicOr(&c.occ[h >> 5], 1u << (h & 31));
}

// ---------------------------------------------------------------------------
// Subtree builder: one CTA per node of level L0 finishes its whole subtree.

// Shared-memory carve-up of k_subtree, in 32-bit words.
constexpr uint32_t ST_OFF_KEYA = 0;
constexpr uint32_t ST_OFF_POSA = ST_OFF_KEYA + ST_CAP;
constexpr uint32_t ST_OFF_KEYB = ST_OFF_POSA + ST_CAP;
constexpr uint32_t ST_OFF_POSB = ST_OFF_KEYB + ST_CAP;
constexpr uint32_t ST_OFF_CNT = ST_OFF_POSB + ST_CAP;
constexpr uint32_t ST_OFF_CNT2 = ST_OFF_CNT + ST_CAP;
constexpr uint32_t ST_OFF_START = ST_OFF_CNT2 + ST_CAP;
constexpr uint32_t ST_OFF_TOPI = ST_OFF_START + ST_CAP + 1;
constexpr uint32_t ST_OFF_WS = ST_OFF_TOPI + ST_CAP;
constexpr uint32_t ST_WORDS = ST_OFF_WS + 33;
constexpr size_t st_smem_bytes() { return (size_t) ST_WORDS * 4; }
static_assert(st_smem_bytes() <= 227 * 1024, "subtree builder shared memory");

template <typename U>
__device__ void block_scan_array(const U *in, U *out, uint32_t n, U *ws)
{
	// out[i] = sum in[0..i); out[n] = total.  in may equal out.
	U carry = 0;
	for (uint32_t b = 0; b < n; b += blockDim.x) {
		const uint32_t i = b + threadIdx.x;
		const U v = i < n ? in[i] : U(0);
		U tot;
		const U ex = block_excl_scan<U>(v, &tot, ws);
		if (i < n)
			out[i] = carry + ex;
		carry += tot;
	}
	if (threadIdx.x == 0)
		out[n] = carry;
	__syncthreads();
}

template <typename T, bool HAS_ID>
__global__ void __launch_bounds__(ST_THREADS) k_subtree(BuildCtx<T, HAS_ID> c, uint32_t L0,
                                                       const uint32_t *__restrict__ B)
{
	extern __shared__ __align__(16) uint32_t st_smem[];
	uint32_t *keyA = st_smem + ST_OFF_KEYA;
	uint32_t *posA = st_smem + ST_OFF_POSA;
	uint32_t *keyB = st_smem + ST_OFF_KEYB;
	uint32_t *posB = st_smem + ST_OFF_POSB;
	uint32_t *cnt = st_smem + ST_OFF_CNT;     // [ST_CAP] counts of the current sub-level
	uint32_t *cnt2 = st_smem + ST_OFF_CNT2;   // [ST_CAP] counts of the next sub-level
	uint32_t *start = st_smem + ST_OFF_START; // [ST_CAP + 1]
	uint32_t *topi = st_smem + ST_OFF_TOPI;   // [ST_CAP]
	uint32_t *ws = st_smem + ST_OFF_WS;       // [33]
	__shared__ uint32_t s_n;

	const uint32_t j = blockIdx.x;
	const uint64_t cN = node_count(c.n, L0, j);
	if (cN == 0)
		return;
	const uint32_t lo = L0 ? B[j] : 0u;
	const uint32_t hi = L0 ? B[j + 1] : (uint32_t) c.n;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = ST_THREADS / 32;

	// Gather the points still free in [lo, hi), in dim1 order.
	if (threadIdx.x == 0)
		s_n = 0;
	__syncthreads();
	for (uint32_t b = lo; b < hi; b += ST_THREADS) {
		const uint32_t i = b + threadIdx.x;
		const uint32_t v = i < hi ? c.r2p1[i] : 0u;
		const uint32_t keep = v != 0;
		uint32_t tot;
		const uint32_t off = block_excl_scan<uint32_t>(keep, &tot, ws);
		const uint32_t base = s_n;
		if (keep && base + off < ST_CAP) {
			keyA[base + off] = v;
			posA[base + off] = i;
		}
		__syncthreads();
		if (threadIdx.x == 0)
			s_n = base + tot;
		__syncthreads();
	}
	if (s_n != cN || cN > ST_CAP) {
		if (threadIdx.x == 0)
			atomicOr(c.err, 2u);
		return;
	}
	const uint32_t h0 = (1u << L0) + j;
	const uint32_t last_s = c.D - 1 - L0;
	const uint32_t half = 1u << (c.D - 1);  // med exists for positions < half
	uint32_t *kc = keyA, *pc = posA, *kn = keyB, *pn = posB;
	uint32_t nsub = 1;
	uint32_t present = (uint32_t) cN;
	if (threadIdx.x == 0)
		cnt[0] = (uint32_t) cN;
	__syncthreads();
	for (uint32_t s = 0;; s++) {
		block_scan_array<uint32_t>(cnt, start, nsub, ws);
		const bool wide = present / nsub >= 64;
		// arg-max of every sub-node (keys are distinct dim2 ranks)
		if (wide) {
			for (uint32_t t = warp; t < nsub; t += nwarps) {
				uint64_t bestv = 0;
				for (uint32_t i = start[t] + lane; i < start[t + 1]; i += 32)
					bestv = max(bestv, ((uint64_t) kc[i] << 32) | i);
#pragma unroll
				for (int o = 16; o > 0; o >>= 1) {
					const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, bestv, o);
					bestv = max(bestv, other);
				}
				if (lane == 0)
					topi[t] = (uint32_t) bestv;
			}
		} else {
			for (uint32_t t = threadIdx.x; t < nsub; t += ST_THREADS) {
				uint32_t bk = 0, bi = 0;
				for (uint32_t i = start[t]; i < start[t + 1]; i++)
					if (kc[i] > bk) {
						bk = kc[i];
						bi = i;
					}
				topi[t] = bi;
			}
		}
		__syncthreads();
		// write the nodes of this sub-level
		for (uint32_t tb = 0; tb < nsub; tb += ST_THREADS) {
			const uint32_t t = tb + threadIdx.x;
			bool occupied = false;
			uint32_t h = 0;
			if (t < nsub) {
				const uint32_t ct = cnt[t];
				h = (h0 << s) + t;
				if (ct > 0) {
					occupied = true;
					const uint32_t ti = topi[t];
					const Point<T, HAS_ID> p = c.point_at(pc[ti]);
					c.write_node(h, p);
					if (h < half) {
						T m = p.dim1;
						if (ct >= 2) {
							uint32_t mi = start[t] + ct / 2 - 1;
							if (ti <= mi)
								mi++;
							m = c.point_at(pc[mi]).dim1;
						}
						c.med[h] = m;
					}
				}
			}
			// occupancy: the lanes of a warp cover one aligned run of <= 32 positions
			const uint32_t bits = __ballot_sync(0xFFFFFFFFu, occupied);
			const uint32_t first = __shfl_sync(0xFFFFFFFFu, h, 0);
			if (lane == 0 && bits) {
				const uint32_t wbase = (h0 << s) + tb + warp * 32;
				if (nsub >= 32)
					atomicOr(&c.occ[wbase >> 5], bits);
				else
					atomicOr(&c.occ[first >> 5], bits << (first & 31));
			}
		}
		if (s == last_s)
			break;
		// counts of the next sub-level
		for (uint32_t t = threadIdx.x; t < nsub; t += ST_THREADS) {
			const uint32_t ct = cnt[t];
			cnt2[2 * t] = ct ? ct / 2 : 0u;
			cnt2[2 * t + 1] = ct ? ct - 1 - ct / 2 : 0u;
		}
		// drop each sub-node's point; every segment is non-empty above the last level
		if (wide) {
			for (uint32_t t = warp; t < nsub; t += nwarps) {
				const uint32_t ti = topi[t];
				for (uint32_t i = start[t] + lane; i < start[t + 1]; i += 32)
					if (i != ti) {
						const uint32_t ni = i - t - (i > ti ? 1u : 0u);
						kn[ni] = kc[i];
						pn[ni] = pc[i];
					}
			}
		} else {
			for (uint32_t t = threadIdx.x; t < nsub; t += ST_THREADS) {
				const uint32_t ti = topi[t];
				for (uint32_t i = start[t]; i < start[t + 1]; i++)
					if (i != ti) {
						const uint32_t ni = i - t - (i > ti ? 1u : 0u);
						kn[ni] = kc[i];
						pn[ni] = pc[i];
					}
			}
		}
		__syncthreads();
		for (uint32_t t = threadIdx.x; t < 2 * nsub; t += ST_THREADS)
			cnt[t] = cnt2[t];
		present -= nsub;
		nsub *= 2;
		uint32_t *tk = kc, *tp = pc;
		kc = kn;
		pc = pn;
		kn = tk;
		pn = tp;
		__syncthreads();
	}
}


template <typename T>
T *as(void *p)
{
	return static_cast<T *>(p);
}

struct DevBuf {
	void *p = nullptr;
	cudaStream_t s = nullptr;
	DevBuf() = default;
	DevBuf(size_t bytes, cudaStream_t st) : s(st)
	{
		if (bytes == 0)
			return;
		cudaError_t e = cudaMallocAsync(&p, bytes, st);
		if (e == cudaErrorMemoryAllocation) {
			cudaGetLastError();
			fail(PST_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " B failed during construction");
		}
		check_cuda(e, "cudaMallocAsync");
	}
	~DevBuf()
	{
		if (p)
			cudaFreeAsync(p, s);
	}
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
	template <typename T>
	T *get() const
	{
		return static_cast<T *>(p);
	}
};

inline unsigned grid_for(uint64_t n, int threads)
{
	const uint64_t want = (n + threads - 1) / threads;
	const uint64_t cap = (uint64_t) device_info().sms * 16;
	return (unsigned) std::max<uint64_t>(1, std::min(want, cap));
}

template <typename T, bool HAS_ID>
void build_impl(TreeStorage &t, const void *pts_d, uint64_t n, cudaStream_t s)
{
	using K = typename KeyOf<T>::K;
	using Pt = Point<T, HAS_ID>;
	const Pt *pts = static_cast<const Pt *>(pts_d);
	const uint32_t D = t.levels;

	// ---- scratch
	const uint64_t rs_tiles = rs_num_tiles(n);
	DevBuf k1(n * sizeof(K), s), k2(n * sizeof(K), s), kalt(n * sizeof(K), s);
	DevBuf valt(n * 4, s), vtmp(n * 4, s), S1b(n * 4, s), Pb(HAS_ID ? n * 4 : 0, s);
	DevBuf tile_hist(256 * rs_tiles * 4, s), scan_tmp(scan_tmp_elems(256 * rs_tiles) * 4, s);
	DevBuf hist_all(8 * 256 * 4, s), flags(64, s);
	uint32_t *hist_host = nullptr;
	PST_CUDA(cudaMallocHost(&hist_host, 8 * 256 * 4));
	struct HostFree {
		uint32_t *p;
		~HostFree() { cudaFreeHost(p); }
	} hf{hist_host};
	SortScratch sc;
	sc.keys_alt = kalt.p;
	sc.vals_alt = valt.get<uint32_t>();
	sc.vals_tmp = vtmp.get<uint32_t>();
	sc.tile_hist = tile_hist.get<uint32_t>();
	sc.scan_tmp = scan_tmp.get<uint32_t>();
	sc.hist_all = hist_all.get<uint32_t>();
	sc.hist_host = hist_host;
	uint32_t *flag = flags.get<uint32_t>();
	PST_CUDA(cudaMemsetAsync(flag, 0, 64, s));

	const unsigned g = grid_for(n, 256);
	// ---- tiebreak order: (id, input index) when ids are not already non-decreasing
	const uint32_t *P = nullptr;
	if constexpr (HAS_ID) {
		k_ids_monotone<T, HAS_ID><<<g, 256, 0, s>>>(pts, n, flag);
		uint32_t mono_flag = 0;
		PST_CUDA(cudaMemcpyAsync(&mono_flag, flag, 4, cudaMemcpyDeviceToHost, s));
		PST_CUDA(cudaStreamSynchronize(s));
		if (mono_flag) {
			uint32_t *idk = reinterpret_cast<uint32_t *>(k1.p);  // k1 is at least n*4 bytes
			k_id_keys<T, HAS_ID><<<g, 256, 0, s>>>(pts, n, idk);
			SortScratch sc32 = sc;
			uint32_t *kres, *vres;
			radix_sort<uint32_t>(idk, nullptr, n, sc32, &kres, &vres, s);
			// vres == null: every digit pass was trivial, i.e. all ids equal; then
			// (id, index) order is index order and P stays the identity.
			if (vres) {
				PST_CUDA(cudaMemcpyAsync(Pb.p, vres, n * 4, cudaMemcpyDeviceToDevice, s));
				P = Pb.get<uint32_t>();
			}
		}
	}
	// ---- dim1 and dim2 orders
	k_value_keys<T, HAS_ID><<<g, 256, 0, s>>>(pts, P, n, k1.get<K>(), k2.get<K>());
	PST_CUDA(cudaGetLastError());
	K *kres;
	uint32_t *vres;
	radix_sort<K>(k1.get<K>(), nullptr, n, sc, &kres, &vres, s);
	// A null payload result means all keys were equal: the order is the identity.
	uint32_t *S1 = S1b.get<uint32_t>();
	if (vres)
		PST_CUDA(cudaMemcpyAsync(S1, vres, n * 4, cudaMemcpyDeviceToDevice, s));
	else
		k_iota<<<g, 256, 0, s>>>(S1, n);
	radix_sort<K>(k2.get<K>(), nullptr, n, sc, &kres, &vres, s);
	if (!vres) {
		vres = valt.get<uint32_t>();
		k_iota<<<g, 256, 0, s>>>(vres, n);
	}
	// vres: dim2-sorted position -> tiebreak rank (S2).  k1's storage is free now.
	uint32_t *rank2_of_tb = reinterpret_cast<uint32_t *>(k1.p);
	k_rank_scatter<<<g, 256, 0, s>>>(vres, n, rank2_of_tb);
	uint32_t *r2p1 = reinterpret_cast<uint32_t *>(kalt.p);
	if (reinterpret_cast<void *>(vres) == kalt.p)
		fail(PST_ERR_INTERNAL, "scratch aliasing");
	uint32_t *pos_of_rank2 = vres == valt.get<uint32_t>() ? vtmp.get<uint32_t>() : valt.get<uint32_t>();
	k_sorted_ranks<<<g, 256, 0, s>>>(S1, rank2_of_tb, n, r2p1, pos_of_rank2);
	PST_CUDA(cudaGetLastError());

	// ---- levels
	const uint32_t L0 = std::min(subtree_level(n), D - 1);
	const uint64_t nodes_wide = 1ull << L0;
	DevBuf Ba((nodes_wide + 1) * 4, s), Bb((nodes_wide + 1) * 4, s), bestb(nodes_wide * 4, s), topb(nodes_wide * 4, s);
	BuildCtx<T, HAS_ID> c;
	c.pts = pts;
	c.P = P;
	c.S1 = S1;
	c.r2p1 = r2p1;
	c.pos_of_rank2 = pos_of_rank2;
	c.dim1 = as<T>(t.dim1);
	c.dim2 = as<T>(t.dim2);
	c.med = as<T>(t.med);
	c.id = t.id;
	c.occ = t.occ;
	c.top_pos = topb.get<uint32_t>();
	c.err = flag + 1;
	c.n = n;
	c.D = D;
	uint32_t *B = Ba.get<uint32_t>(), *Bn = Bb.get<uint32_t>();
	{
		const uint32_t b0[2] = {0u, (uint32_t) n};
		PST_CUDA(cudaMemcpyAsync(B, b0, 8, cudaMemcpyHostToDevice, s));
	}
	const uint64_t am_tiles = (n + AM_TILE - 1) / AM_TILE;
	const uint64_t am_ctas_max = (uint64_t) device_info().sms * 8;
	const uint64_t tiles_per_cta = (am_tiles + am_ctas_max - 1) / am_ctas_max;
	const unsigned am_grid = (unsigned) ((am_tiles + tiles_per_cta - 1) / tiles_per_cta);
	for (uint32_t d = 0; d < L0; d++) {
		const uint32_t nseg = 1u << d;
		PST_CUDA(cudaMemsetAsync(bestb.p, 0, nseg * 4, s));
		k_level_argmax<<<am_grid, AM_THREADS, 0, s>>>(r2p1, n, B, nseg, bestb.get<uint32_t>(), tiles_per_cta);
		k_level_nodes<T, HAS_ID><<<(nseg + 127) / 128, 128, 0, s>>>(c, d, B, Bn, bestb.get<uint32_t>());
		PST_CUDA(cudaGetLastError());
		std::swap(B, Bn);
	}
	PST_CUDA(cudaFuncSetAttribute(k_subtree<T, HAS_ID>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                              (int) st_smem_bytes()));
	k_subtree<T, HAS_ID><<<(unsigned) nodes_wide, ST_THREADS, st_smem_bytes(), s>>>(c, L0, B);
	PST_CUDA(cudaGetLastError());
	uint32_t errs[2] = {0, 0};
	PST_CUDA(cudaMemcpyAsync(errs, flag, 8, cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaStreamSynchronize(s));
	if (errs[1])
		fail(PST_ERR_INTERNAL, "construction consistency check failed (code " + std::to_string(errs[1]) + ")");
}

}  // namespace

uint64_t tree_bytes(pst_dtype dt, pst_idtype it, uint64_t n) { return tree_layout(dt, it, n).total; }

uint64_t build_bytes_needed(pst_dtype dt, pst_idtype it, uint64_t n)
{
	const uint64_t ks = value_size(dt);
	const uint64_t tiles = rs_num_tiles(n);
	const uint64_t wide = 1ull << subtree_level(n);
	const uint64_t scratch = n * (3 * ks + 3 * 4 + (it == PST_ID_U32 ? 4 : 0)) + 256 * tiles * 4 +
	                         scan_tmp_elems(256 * tiles) * 4 + wide * 16 + (1 << 20);
	return tree_bytes(dt, it, n) + scratch;
}

void build_tree(TreeStorage &t, const void *pts_d, uint64_t n, cudaStream_t s)
{
	if (n >= (1ull << 31))
		fail(PST_ERR_INVALID, "at most 2^31 - 1 points per tree");
	t.n = n;
	t.levels = tree_levels(n);
	if (n == 0)
		return;
	if (!pts_d)
		fail(PST_ERR_INVALID, "null point array");
	const TreeLayout L = tree_layout(t.dtype, t.idtype, n);
	cudaError_t e = cudaMalloc(&t.mem, L.total);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		fail(PST_ERR_NOMEM, "tree allocation of " + std::to_string(L.total) + " B failed");
	}
	check_cuda(e, "cudaMalloc(tree)");
	t.bytes = L.total;
	char *b = static_cast<char *>(t.mem);
	t.dim1 = b + L.off_dim1;
	t.dim2 = b + L.off_dim2;
	t.med = b + L.off_med;
	t.id = t.idtype == PST_ID_U32 ? reinterpret_cast<uint32_t *>(b + L.off_id) : nullptr;
	t.occ = reinterpret_cast<uint32_t *>(b + L.off_occ);
	PST_CUDA(cudaMemsetAsync(t.occ, 0, L.total - L.off_occ, s));
	try {
		switch (t.dtype) {
		case PST_F32:
			t.idtype == PST_ID_U32 ? build_impl<float, true>(t, pts_d, n, s) : build_impl<float, false>(t, pts_d, n, s);
			break;
		case PST_F64:
			t.idtype == PST_ID_U32 ? build_impl<double, true>(t, pts_d, n, s) : build_impl<double, false>(t, pts_d, n, s);
			break;
		case PST_I32:
			t.idtype == PST_ID_U32 ? build_impl<int32_t, true>(t, pts_d, n, s) : build_impl<int32_t, false>(t, pts_d, n, s);
			break;
		}
		PST_CUDA(cudaStreamSynchronize(s));
	} catch (...) {
		cudaStreamSynchronize(s);
		cudaFree(t.mem);
		t.mem = nullptr;
		throw;
	}
}

void free_tree(TreeStorage &t)
{
	if (t.mem)
		cudaFree(t.mem);
	t.mem = nullptr;
}

void export_tree(const TreeStorage &t, void *dim1, void *dim2, void *med, uint32_t *ids, uint8_t *bitcodes)
{
	if (t.n == 0)
		return;
	const uint32_t D = t.levels;
	const uint64_t S = 1ull << D;  // positions 0..S-1, position 0 unused
	const size_t vs = value_size(t.dtype);
	std::vector<unsigned char> h1(S * vs), h2(S * vs), hm((S / 2) * vs);
	std::vector<uint32_t> hid(t.id ? S : 0), hocc(std::max<uint64_t>(S / 32, 1));
	PST_CUDA(cudaMemcpy(h1.data(), t.dim1, S * vs, cudaMemcpyDeviceToHost));
	PST_CUDA(cudaMemcpy(h2.data(), t.dim2, S * vs, cudaMemcpyDeviceToHost));
	PST_CUDA(cudaMemcpy(hm.data(), t.med, (S / 2) * vs, cudaMemcpyDeviceToHost));
	if (t.id)
		PST_CUDA(cudaMemcpy(hid.data(), t.id, S * 4, cudaMemcpyDeviceToHost));
	PST_CUDA(cudaMemcpy(hocc.data(), t.occ, hocc.size() * 4, cudaMemcpyDeviceToHost));
	auto occ = [&](uint64_t h) { return h < S && ((hocc[h >> 5] >> (h & 31)) & 1u); };
	unsigned char *o1 = static_cast<unsigned char *>(dim1), *o2 = static_cast<unsigned char *>(dim2),
	              *om = static_cast<unsigned char *>(med);
	for (uint64_t h = 1; h < S; h++) {
		const uint64_t slot = h - 1;
		if (!occ(h)) {
			memset(o1 + slot * vs, 0, vs);
			memset(o2 + slot * vs, 0, vs);
			memset(om + slot * vs, 0, vs);
			if (ids)
				ids[slot] = 0;
			bitcodes[slot] = 0;
			continue;
		}
		memcpy(o1 + slot * vs, &h1[h * vs], vs);
		memcpy(o2 + slot * vs, &h2[h * vs], vs);
		// last-level nodes are leaves; a leaf's median is its own dim1
		// (pst/static-pst-cpu-iter.tpp:512-517)
		memcpy(om + slot * vs, h < S / 2 ? &hm[h * vs] : &h1[h * vs], vs);
		if (ids)
			ids[slot] = t.id ? hid[h] : 0;
		bitcodes[slot] = (uint8_t) ((occ(2 * h) ? 0x2 : 0) | (occ(2 * h + 1) ? 0x1 : 0));
	}
}

}  // namespace pst
