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
//   1. every point gets a tiebreak rank tb (its place in (id, input index) order) and
//      a 64-bit dim2 key whose order is the dim2 order: (dim2 key << 32 | tb + 1) for
//      4-byte values, (dim2 rank << 32 | tb + 1) for doubles (one extra sort finds
//      the ranks).  One radix sort by dim1 key carries these keys along, so position
//      i of the sorted arrays is the i-th point in dim1 order;
//   2. for the wide top levels, a segmented arg-max over the sorted dim2 keys picks
//      every node's point of the level at once.  It reads a maximum per 512-position
//      tile and scans only the tiles cut by a node boundary; points taken by
//      ancestors are marked in a bitmap, and only the tiles that lost a point are
//      re-reduced.  A per-node kernel then finds the taken point's position (binary
//      search on (dim1 key, tb)) and places the median;
//   3. once every node of a level holds at most ST_CAP points, one CTA per node
//      builds the whole remaining subtree in shared memory.
#include <algorithm>
#include <limits>
#include <type_traits>
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

// Subtree builder capacity: nodes of at most ST_CAP points are finished by one CTA
// (a power of two; PST_SUBTREE_CAP overrides it at build time).
#ifndef PST_SUBTREE_CAP
#define PST_SUBTREE_CAP 512
#endif
constexpr uint32_t ST_CAP = PST_SUBTREE_CAP;
constexpr int ST_THREADS = 256;
// Arg-max tiles: every segment of a level before the subtree level spans at least
// ST_CAP >= TM_TILE positions, so a tile is cut by at most one segment boundary.
constexpr uint32_t TM_TILE = ST_CAP < 512 ? ST_CAP : 512;
constexpr int AM_THREADS = 256;
static_assert(ST_CAP >= TM_TILE, "tile/segment invariant");
static_assert(TM_TILE % 32 == 0, "tiles are whole bitmap words");

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

// Sorted arrays, position i = i-th point in dim1 order:
//   k1s[i]  dim1 key, c2s[i] 64-bit dim2 key (never 0; low 32 bits = tb + 1),
//   taken   one bit per position, set once the point is stored in a node.
template <typename T, bool HAS_ID>
struct BuildCtx {
	using K = typename KeyOf<T>::K;
	const Point<T, HAS_ID> *pts;
	const uint32_t *P;  // tiebreak rank -> input index (null: identity)
	const K *k1s;
	const uint64_t *c2s;
	uint32_t *taken;
	uint64_t *tmax;     // per TM_TILE tile: max c2s over positions not taken (0 if none)
	T *dim1;
	T *dim2;
	T *med;
	uint32_t *id;
	uint32_t *occ;
	uint32_t *top_pos;  // heap position -> dim1-sorted position of its point (levels < L0)
	uint32_t *err;
	uint64_t n;
	uint32_t D;
	// Points are rebuilt from their sorted keys instead of gathered from the input:
	// set for 4-byte values when no value is -0.0 (the only value the keys do not
	// keep: it shares +0.0's key) and the ids, if any, equal the input indices (so
	// the id is the tiebreak rank the dim2 key carries).
	bool recon;

	__device__ __forceinline__ Point<T, HAS_ID> point_of_tb(uint32_t tb) const { return pts[P ? P[tb] : tb]; }
	__device__ __forceinline__ static uint32_t tb_of(uint64_t key2) { return (uint32_t) key2 - 1u; }
	// The point of dim1 key k1 and 64-bit dim2 key c2 (recon only).
	__device__ __forceinline__ static Point<T, HAS_ID> point_from_keys(K k1, uint64_t c2)
	{
		Point<T, HAS_ID> p;
		p.dim1 = KeyOf<T>::value(k1);
		p.dim2 = KeyOf<T>::value((K) (c2 >> 32));
		if constexpr (HAS_ID)
			p.id = tb_of(c2);
		return p;
	}
	__device__ __forceinline__ Point<T, HAS_ID> point_at(uint32_t pos) const
	{
		if constexpr (sizeof(K) == 4) {
			if (recon)
				return point_from_keys(k1s[pos], c2s[pos]);
		}
		return point_of_tb(tb_of(c2s[pos]));
	}
	__device__ __forceinline__ bool is_taken(uint64_t pos) const { return (taken[pos >> 5] >> (pos & 31)) & 1u; }

	__device__ __forceinline__ void write_node(uint32_t h, const Point<T, HAS_ID> &p) const
	{
		dim1[h] = p.dim1;
		dim2[h] = p.dim2;
		if constexpr (HAS_ID)
			id[h] = p.id;
	}
};

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const uint64_t t = __shfl_xor_sync(0xFFFFFFFFu, v, o);
		v = t > v ? t : v;
	}
	return v;
}

template <typename K>
__device__ __forceinline__ void atomic_min_key(K *p, K v)
{
	if constexpr (sizeof(K) == 4)
		atomicMin(reinterpret_cast<unsigned int *>(p), (unsigned int) v);
	else
		atomicMin(reinterpret_cast<unsigned long long *>(p), (unsigned long long) v);
}

template <typename K>
__device__ __forceinline__ void atomic_max_key(K *p, K v)
{
	if constexpr (sizeof(K) == 4)
		atomicMax(reinterpret_cast<unsigned int *>(p), (unsigned int) v);
	else
		atomicMax(reinterpret_cast<unsigned long long *>(p), (unsigned long long) v);
}

// Block-wide min and max of (lo, hi), folded into range[0] / range[1] with atomics.
template <typename K>
__device__ void block_range_fold(K lo, K hi, K *range)
{
	__shared__ K s_lo[32], s_hi[32];
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const K a = __shfl_xor_sync(0xFFFFFFFFu, lo, o), b = __shfl_xor_sync(0xFFFFFFFFu, hi, o);
		lo = a < lo ? a : lo;
		hi = b > hi ? b : hi;
	}
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
	if (lane == 0) {
		s_lo[warp] = lo;
		s_hi[warp] = hi;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int w = 1; w < nw; w++) {
			lo = s_lo[w] < lo ? s_lo[w] : lo;
			hi = s_hi[w] > hi ? s_hi[w] : hi;
		}
		atomic_min_key<K>(&range[0], lo);
		atomic_max_key<K>(&range[1], hi);
	}
}

// ---------------------------------------------------------------------------
// Preparation kernels.

template <typename T, bool HAS_ID>
__global__ void k_id_keys(const Point<T, HAS_ID> *pts, uint64_t n, uint32_t *keys)
{
	if constexpr (HAS_ID) {
		for (uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t) gridDim.x * blockDim.x)
			keys[i] = pts[i].id;
	}
}

// Copies of the digit histogram a block of k_prep_keys keeps in shared memory (a
// quarter of its warps on each), so that keys sharing a digit meet on fewer counters.
constexpr int PK_HIST_COPIES = 4;

// Keys in tiebreak-rank order r (input index P[r]): k1[r] = dim1 key and either the
// final 64-bit dim2 key (4-byte values) or the raw dim2 key k2[r] (doubles).
// range = [min k1, max k1, min k2, max k2]; *negzero |= 1 when a value is -0.0 (the
// one value its key does not keep).
// SCAN_IDS (P null, points with ids): the same pass checks the ids, idflag |= 1 when
// they decrease somewhere and |= 2 when some id differs from its input index,
// id_range = [min id, max id].  hist (non-null): the pass also counts the 8-bit
// digits of the dim1 keys, hist[d * 256 + v] += keys whose digit d is v, for every
// digit of the key (the radix sort's histogram, which the order of the keys does
// not change); dynamic shared memory PK_HIST_COPIES * sizeof(K) * 256 words.
template <typename T, bool HAS_ID, bool SCAN_IDS>
__global__ void k_prep_keys(const Point<T, HAS_ID> *pts, const uint32_t *P, uint64_t n,
                            typename KeyOf<T>::K *k1, uint64_t *c2, typename KeyOf<T>::K *k2,
                            typename KeyOf<T>::K *range, uint32_t *negzero, uint32_t *idflag,
                            uint32_t *id_range, uint32_t *hist)
{
	using K = typename KeyOf<T>::K;
	constexpr int ND = (int) sizeof(K);  // 8-bit digits of a key
	extern __shared__ uint32_t pk_hist[];
	uint32_t *myh = pk_hist + ((threadIdx.x >> 5) % PK_HIST_COPIES) * (ND * 256);
	if (hist) {
		for (int i = threadIdx.x; i < PK_HIST_COPIES * ND * 256; i += blockDim.x)
			pk_hist[i] = 0;
		__syncthreads();
	}
	K lo1 = ~K(0), hi1 = 0, lo2 = ~K(0), hi2 = 0;
	bool nz = false;
	uint32_t ilo = 0xFFFFFFFFu, ihi = 0;
	bool dec = false, other = false;
	for (uint64_t r = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t) gridDim.x * blockDim.x) {
		const Point<T, HAS_ID> p = pts[P ? P[r] : r];
		if constexpr (SCAN_IDS && HAS_ID) {
			const uint32_t v = p.id;
			ilo = min(ilo, v);
			ihi = max(ihi, v);
			if (r + 1 < n && v > pts[r + 1].id)
				dec = true;
			if ((uint64_t) v != r)
				other = true;
		}
		const K a = KeyOf<T>::key(p.dim1), b = KeyOf<T>::key(p.dim2);
		if constexpr (!std::is_integral<T>::value)
			nz |= (p.dim1 == T(0) && signbit(p.dim1)) || (p.dim2 == T(0) && signbit(p.dim2));
		k1[r] = a;
		if constexpr (sizeof(K) == 4)
			c2[r] = ((uint64_t) b << 32) | (uint64_t) (r + 1);
		else
			k2[r] = b;
		if (hist) {
#pragma unroll
			for (int d = 0; d < ND; d++)
				atomicAdd(&myh[d * 256 + (uint32_t) ((a >> (8 * d)) & 0xFFu)], 1u);
		}
		lo1 = a < lo1 ? a : lo1;
		hi1 = a > hi1 ? a : hi1;
		lo2 = b < lo2 ? b : lo2;
		hi2 = b > hi2 ? b : hi2;
	}
	if (__any_sync(0xFFFFFFFFu, nz) && (threadIdx.x & 31) == 0)
		atomicOr(negzero, 1u);
	if constexpr (SCAN_IDS && HAS_ID) {
		if (__any_sync(0xFFFFFFFFu, dec) && (threadIdx.x & 31) == 0)
			atomicOr(idflag, 1u);
		if (__any_sync(0xFFFFFFFFu, other) && (threadIdx.x & 31) == 0)
			atomicOr(idflag, 2u);
		block_range_fold<uint32_t>(ilo, ihi, id_range);
		__syncthreads();
	}
	block_range_fold<K>(lo1, hi1, range);
	__syncthreads();
	block_range_fold<K>(lo2, hi2, range + 2);
	if (hist) {
		__syncthreads();
		for (int i = threadIdx.x; i < ND * 256; i += blockDim.x) {
			uint32_t t = 0;
#pragma unroll
			for (int c = 0; c < PK_HIST_COPIES; c++)
				t += pk_hist[c * ND * 256 + i];
			if (t)
				atomicAdd(&hist[i], t);
		}
	}
}

// Doubles: S2 = dim2-sorted position -> tb (null: identity); c2[tb] = rank << 32 | tb + 1.
__global__ void k_rank_keys(const uint32_t *S2, uint64_t n, uint64_t *c2)
{
	for (uint64_t j = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t) gridDim.x * blockDim.x) {
		const uint32_t tb = S2 ? S2[j] : (uint32_t) j;
		c2[tb] = (j << 32) | (uint64_t) (tb + 1);
	}
}

// ---------------------------------------------------------------------------
// Wide levels.

// Maximum of c2s over the positions of tile t that are not taken; one warp per tile.
__device__ __forceinline__ uint64_t tile_max(const uint64_t *__restrict__ c2s, const uint32_t *__restrict__ taken,
                                             uint64_t n, uint64_t t)
{
	const uint32_t lane = lane_id();
	const uint64_t t0 = t * TM_TILE;
	uint64_t m = 0;
#pragma unroll 4
	for (uint32_t k = 0; k < TM_TILE / 32; k++) {
		const uint64_t i = t0 + k * 32 + lane;
		if (i < n) {
			const uint32_t w = taken[i >> 5];  // one word per k, the same for the whole warp
			if (!((w >> lane) & 1u))
				m = max(m, c2s[i]);
		}
	}
	return warp_max_u64(m);
}

__global__ void __launch_bounds__(AM_THREADS) k_tile_max_all(const uint64_t *__restrict__ c2s,
                                                             const uint32_t *__restrict__ taken, uint64_t n,
                                                             uint64_t *tmax)
{
	const uint64_t ntiles = (n + TM_TILE - 1) / TM_TILE;
	const uint64_t gw = ((uint64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nw = ((uint64_t) gridDim.x * blockDim.x) >> 5;
	for (uint64_t t = gw; t < ntiles; t += nw) {
		const uint64_t m = tile_max(c2s, taken, n, t);
		if (lane_id() == 0)
			tmax[t] = m;
	}
}

// Re-reduces the tiles that lost a point at level d (one warp per node).
__global__ void __launch_bounds__(AM_THREADS) k_tile_refresh(const uint64_t *__restrict__ c2s,
                                                             const uint32_t *__restrict__ taken, uint64_t n,
                                                             const uint32_t *__restrict__ top_pos, uint32_t d,
                                                             uint64_t *tmax, const uint32_t *err)
{
	const uint32_t nseg = 1u << d;
	const uint64_t gw = ((uint64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (gw >= nseg || *err)  // after an error top_pos may hold unwritten entries
		return;
	const uint64_t t = top_pos[nseg + gw] / TM_TILE;
	if (t >= (n + TM_TILE - 1) / TM_TILE)
		return;
	const uint64_t m = tile_max(c2s, taken, n, t);
	if (lane_id() == 0)
		tmax[t] = m;  // tiles shared by two nodes get the same value twice
}

// best[s] = max c2s over the positions of [B[s], B[s+1]) not taken.  A thread owns a
// tile: tiles inside one segment contribute their tmax (one atomic per run of equal
// segments in a warp); a tile cut by a boundary is scanned by the whole warp.
__global__ void __launch_bounds__(AM_THREADS) k_level_argmax(const uint64_t *__restrict__ c2s,
                                                             const uint32_t *__restrict__ taken,
                                                             const uint64_t *__restrict__ tmax, uint64_t n,
                                                             const uint32_t *__restrict__ B, uint32_t nseg,
                                                             unsigned long long *best, const uint32_t *err,
                                                             float seg_per_pos)
{
	if (*err)  // after an error the bounds may hold unwritten entries
		return;
	const uint64_t ntiles = (n + TM_TILE - 1) / TM_TILE;
	const uint32_t lane = lane_id();
	const uint64_t gw = ((uint64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint64_t nw = ((uint64_t) gridDim.x * blockDim.x) >> 5;
	for (uint64_t wb = gw * 32; wb < ntiles; wb += nw * 32) {
		const uint64_t t = wb + lane;
		const bool valid = t < ntiles;
		const uint64_t t0 = t * TM_TILE;
		const uint64_t t1 = valid ? min(t0 + TM_TILE, n) : 0;
		uint32_t seg = 0xFFFFFFFFu;
		uint64_t seg_end = 0;
		if (valid) {
			// the largest s with B[s] <= t0: the level's segments are all within a few
			// positions of n / nseg long, so s lies next to t0 * nseg / n and a short
			// walk from there finds it (B increases, B[0] = 0)
			uint32_t g = min((uint32_t) ((float) t0 * seg_per_pos), nseg - 1);
			while (g > 0 && B[g] > t0)
				g--;
			while (g + 1 < nseg && B[g + 1] <= t0)
				g++;
			seg = g;
			seg_end = B[g + 1];
		}
		const bool whole = valid && t1 <= seg_end;
		uint64_t v = whole ? tmax[t] : 0;
		// max over runs of equal segments (segments do not decrease along the lanes)
		const uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, seg, 1);
		const uint32_t heads = __ballot_sync(0xFFFFFFFFu, lane == 0 || prev != seg);
		const uint32_t start = 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint64_t u = __shfl_up_sync(0xFFFFFFFFu, v, o);
			if (lane >= start + o)
				v = u > v ? u : v;
		}
		const uint32_t next = __shfl_down_sync(0xFFFFFFFFu, seg, 1);
		if (valid && (lane == 31 || next != seg) && v)
			atomicMax(&best[seg], (unsigned long long) v);
		// tiles cut by a boundary: positions below seg_end belong to seg, the rest to seg + 1
		uint32_t cut = __ballot_sync(0xFFFFFFFFu, valid && !whole);
		while (cut) {
			const int src = __ffs(cut) - 1;
			cut &= cut - 1;
			const uint64_t c0 = __shfl_sync(0xFFFFFFFFu, t0, src);
			const uint64_t c1 = __shfl_sync(0xFFFFFFFFu, t1, src);
			const uint64_t ce = __shfl_sync(0xFFFFFFFFu, seg_end, src);
			const uint32_t cs = __shfl_sync(0xFFFFFFFFu, seg, src);
			uint64_t ma = 0, mb = 0;
#pragma unroll 4
			for (uint32_t k = 0; k < TM_TILE / 32; k++) {
				const uint64_t i = c0 + k * 32 + lane;
				if (i < c1) {
					const uint32_t w = taken[i >> 5];
					if (!((w >> lane) & 1u)) {
						const uint64_t x = c2s[i];
						if (i < ce)
							ma = max(ma, x);
						else
							mb = max(mb, x);
					}
				}
			}
			ma = warp_max_u64(ma);
			mb = warp_max_u64(mb);
			if (lane == 0) {
				if (ma)
					atomicMax(&best[cs], (unsigned long long) ma);
				if (mb)
					atomicMax(&best[cs + 1], (unsigned long long) mb);
			}
		}
	}
}

// One thread per node of level d: locate the arg-max point, place the median, write
// the node and the next level's segment bounds.  Bounds are dim1-sorted positions
// that still include points taken by ancestors; those (at most d of them inside a
// segment, each the point of one ancestor) are skipped when counting to the median.
template <typename T, bool HAS_ID>
__global__ void k_level_nodes(BuildCtx<T, HAS_ID> c, uint32_t d, const uint32_t *__restrict__ B,
                              uint32_t *__restrict__ Bn, const unsigned long long *__restrict__ best)
{
	using K = typename KeyOf<T>::K;
	const uint32_t nseg = 1u << d;
	const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nseg)
		return;
	if (*c.err)
		return;
	const uint32_t h = nseg + j;
	const uint64_t cnt = node_count(c.n, d, j);
	const uint32_t lo = B[j], hi = B[j + 1];
	const uint64_t bj = best[j];
	if (bj == 0 || cnt < 2 || lo >= hi || hi > c.n) {
		atomicOr(c.err, 1u);
		return;
	}
	// position of the point: first position in [lo, hi) at or after (its dim1 key, tb)
	const uint32_t tb = BuildCtx<T, HAS_ID>::tb_of(bj);
	// the winner's dim1 key (needed to find its position) is known only from its
	// point: one gather per node of the level
	const Point<T, HAS_ID> top = c.point_of_tb(tb);
	const K key1 = KeyOf<T>::key(top.dim1);
	uint32_t a = lo, b = hi;
	while (a < b) {
		const uint32_t mid = a + (b - a) / 2;
		const K km = c.k1s[mid];
		if (km < key1 || (km == key1 && BuildCtx<T, HAS_ID>::tb_of(c.c2s[mid]) < tb))
			a = mid + 1;
		else
			b = mid;
	}
	const uint32_t tp = a;
	if (tp >= hi || c.c2s[tp] != bj) {
		atomicOr(c.err, 8u);
		return;
	}
	atomicOr(&c.taken[tp >> 5], 1u << (tp & 31));
	c.top_pos[h] = tp;
	uint32_t rem[33];
	uint32_t nr = 0;
	rem[nr++] = tp;
	for (uint32_t an = h >> 1; an >= 1; an >>= 1) {
		const uint32_t ta = c.top_pos[an];
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
	c.write_node(h, top);
	c.med[h] = c.point_at(pos).dim1;
	atomicOr(&c.occ[h >> 5], 1u << (h & 31));
}

// ---------------------------------------------------------------------------
// Subtree builder: one CTA per node of level L0 finishes its whole subtree.  The
// CTA holds the 64-bit dim2 keys of its points in dim1 order, each with the slot
// of its point in a shared-memory copy of the subtree's points (gathered once, all
// reads in flight together), so node writes never wait on global memory.

// Shared-memory carve-up of k_subtree, in bytes: points first (8-byte aligned for
// doubles), then the u64 keys, the u16 point slots, the u16 sub-node of every key
// and the u16 arg-max per sub-node.
template <typename T, bool HAS_ID>
struct SubtreeSmem {
	static constexpr size_t PTS = 0;
	static constexpr size_t KEYA = PTS + (size_t) ST_CAP * sizeof(Point<T, HAS_ID>);
	static constexpr size_t KEYB = KEYA + (size_t) ST_CAP * 8;
	static constexpr size_t SLOTA = KEYB + (size_t) ST_CAP * 8;
	static constexpr size_t SLOTB = SLOTA + (size_t) ST_CAP * 2;
	static constexpr size_t SEGA = SLOTB + (size_t) ST_CAP * 2;
	static constexpr size_t SEGB = SEGA + (size_t) ST_CAP * 2;
	static constexpr size_t TOPI = SEGB + (size_t) ST_CAP * 2;
	static constexpr size_t CNT = TOPI + (size_t) ST_CAP * 2;
	static constexpr size_t START = CNT + (size_t) ST_CAP * 2;
	static constexpr size_t WS = START + (size_t) ST_CAP * 2;
	static constexpr size_t BYTES = WS + 33 * 4;
	static_assert(KEYA % 8 == 0 && BYTES <= 227 * 1024, "subtree builder shared memory");
};

// Chunks of ST_THREADS positions the key gather reads: a node's range holds its
// cN <= ST_CAP free points and at most one point taken by each ancestor (< 32).
constexpr int ST_GATHER = (ST_CAP + ST_THREADS - 1) / ST_THREADS + 1;

// Count and start of every sub-node of the current sub-level (in that sub-level's
// compacted key order) are kept in shared memory and derived level to level
// without a scan: going down one level removes each node's point (every node
// above the last level holds one), the left child keeps the first floor(c/2) of
// the rest and the right child the others, so
//   start(2t) = start(t) - t,  start(2t+1) = start(t) - t + floor(c/2).

// The node count of node_count in 32 bits (trees hold fewer than 2^31 points).
__device__ __forceinline__ uint32_t node_count32(uint32_t n, uint32_t d, uint32_t j)
{
	uint32_t c = n;
	for (int b = (int) d - 1; b >= 0 && c != 0; b--)
		c = ((j >> b) & 1u) ? c - 1u - (c >> 1) : c >> 1;
	return c;
}

// Sub-node counts and warps come in powers of two: every quotient in the builder is
// a shift (a run-time divisor costs a division sequence per use, and the builder is
// bound by its instruction issue).
constexpr int ST_LOG_WARPS = 3;
static_assert(ST_THREADS == 32 << ST_LOG_WARPS, "k_subtree: 8 warps");

template <typename T, bool HAS_ID>
__global__ void __launch_bounds__(ST_THREADS) k_subtree(BuildCtx<T, HAS_ID> c, uint32_t L0,
                                                       const uint32_t *__restrict__ B)
{
	using SM = SubtreeSmem<T, HAS_ID>;
	using Pt = Point<T, HAS_ID>;
	extern __shared__ __align__(16) unsigned char st_smem[];
	Pt *spts = reinterpret_cast<Pt *>(st_smem + SM::PTS);
	uint64_t *kc = reinterpret_cast<uint64_t *>(st_smem + SM::KEYA);
	uint64_t *kn = reinterpret_cast<uint64_t *>(st_smem + SM::KEYB);
	uint16_t *sc = reinterpret_cast<uint16_t *>(st_smem + SM::SLOTA);
	uint16_t *sn = reinterpret_cast<uint16_t *>(st_smem + SM::SLOTB);
	uint16_t *gc = reinterpret_cast<uint16_t *>(st_smem + SM::SEGA);     // sub-node of each key
	uint16_t *gn = reinterpret_cast<uint16_t *>(st_smem + SM::SEGB);
	uint16_t *topi = reinterpret_cast<uint16_t *>(st_smem + SM::TOPI);    // [ST_CAP]
	uint16_t *scnt = reinterpret_cast<uint16_t *>(st_smem + SM::CNT);     // [ST_CAP]
	uint16_t *sstart = reinterpret_cast<uint16_t *>(st_smem + SM::START); // [ST_CAP]
	uint32_t *ws = reinterpret_cast<uint32_t *>(st_smem + SM::WS);        // [33]
	__shared__ uint32_t s_pre[ST_GATHER][ST_THREADS / 32];
	__shared__ uint64_t s_pk[ST_THREADS / 32];
	__shared__ uint32_t s_pi[ST_THREADS / 32];
	__shared__ uint32_t s_n;

	const uint32_t j = blockIdx.x;
	const uint32_t cN = node_count32((uint32_t) c.n, L0, j);
	if (cN == 0 || *c.err)
		return;
	const uint32_t lo = L0 ? B[j] : 0u;
	const uint32_t hi = L0 ? B[j + 1] : (uint32_t) c.n;
	if (lo >= hi || hi > c.n || cN > ST_CAP || hi - lo > (uint32_t) (ST_GATHER * ST_THREADS)) {
		if (threadIdx.x == 0)
			atomicOr(c.err, 16u);
		return;
	}
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = ST_THREADS / 32;

	// Gather the keys of the points still free in [lo, hi), in dim1 order: every
	// read in flight at once, then one prefix over (chunk, warp).
	using K = typename BuildCtx<T, HAS_ID>::K;
	// with rebuilt points the dim1 keys come along (contiguous, like the dim2 keys),
	// staged in kn, which the sub-levels only use later
	constexpr bool KEYS4 = sizeof(K) == 4;
	K *k1c = reinterpret_cast<K *>(kn);
	{
		uint64_t v[ST_GATHER];
		K v1[ST_GATHER];
		uint32_t m[ST_GATHER], tw[ST_GATHER];
		// the keys are read with the taken bits, not after them: one round trip
#pragma unroll
		for (int u = 0; u < ST_GATHER; u++) {
			const uint32_t i = lo + (uint32_t) u * ST_THREADS + threadIdx.x;
			const bool in = i < hi;
			tw[u] = in ? c.taken[i >> 5] : 0u;
			v[u] = in ? c.c2s[i] : 0;
			v1[u] = (KEYS4 && c.recon && in) ? c.k1s[i] : K(0);
		}
#pragma unroll
		for (int u = 0; u < ST_GATHER; u++) {
			const uint32_t i = lo + (uint32_t) u * ST_THREADS + threadIdx.x;
			const bool keep = i < hi && !((tw[u] >> (i & 31)) & 1u);
			m[u] = __ballot_sync(0xFFFFFFFFu, keep);
			if (lane == 0)
				s_pre[u][warp] = __popc(m[u]);
		}
		__syncthreads();
		if (warp == 0) {
			// (chunk, warp) pairs in order; lane l sums pairs [l * PER, l * PER + PER)
			constexpr int PAIRS = ST_GATHER * (ST_THREADS / 32), PER = (PAIRS + 31) / 32;
			uint32_t *flat = &s_pre[0][0];
			uint32_t loc[PER], sum = 0;
#pragma unroll
			for (int k = 0; k < PER; k++) {
				const int q = lane * PER + k;
				loc[k] = q < PAIRS ? flat[q] : 0u;
				sum += loc[k];
			}
			const uint32_t inc = warp_incl_scan(sum);
			uint32_t run = inc - sum;
#pragma unroll
			for (int k = 0; k < PER; k++) {
				const int q = lane * PER + k;
				if (q < PAIRS)
					flat[q] = run;
				run += loc[k];
			}
			if (lane == 31)
				s_n = inc;
		}
		__syncthreads();
#pragma unroll
		for (int u = 0; u < ST_GATHER; u++) {
			if ((m[u] >> lane) & 1u) {
				const uint32_t pos = s_pre[u][warp] + __popc(m[u] & lanemask_lt());
				if (pos < ST_CAP) {
					kc[pos] = v[u];
					sc[pos] = (uint16_t) pos;
					gc[pos] = 0;
					if (KEYS4 && c.recon)
						k1c[pos] = v1[u];
				}
			}
		}
	}
	__syncthreads();
	if (s_n != cN) {
		if (threadIdx.x == 0)
			atomicOr(c.err, 2u);
		return;
	}
	// ... and their points: rebuilt from the keys when they can be (no global read
	// at all), otherwise gathered from the input, every read of the CTA in flight at
	// once (one random 12- or 24-byte read per point)
	{
		constexpr int PER = (ST_CAP + ST_THREADS - 1) / ST_THREADS;
		Pt tmp[PER];
#pragma unroll
		for (int u = 0; u < PER; u++) {
			const uint32_t i = threadIdx.x + u * ST_THREADS;
			if (i < cN) {
				if (KEYS4 && c.recon)
					tmp[u] = BuildCtx<T, HAS_ID>::point_from_keys(k1c[i], kc[i]);
				else
					tmp[u] = c.point_of_tb(BuildCtx<T, HAS_ID>::tb_of(kc[i]));
			}
		}
#pragma unroll
		for (int u = 0; u < PER; u++) {
			const uint32_t i = threadIdx.x + u * ST_THREADS;
			if (i < cN)
				spts[i] = tmp[u];
		}
	}
	__syncthreads();
	const uint32_t h0 = (1u << L0) + j;
	const uint32_t last_s = c.D - 1 - L0;
	const uint32_t half = 1u << (c.D - 1);  // med exists for positions < half
	uint32_t present = cN;
	if (threadIdx.x == 0) {
		scnt[0] = (uint16_t) cN;
		sstart[0] = 0;
	}
	__syncthreads();
	for (uint32_t s = 0;; s++) {
		const uint32_t nsub = 1u << s;
		const bool wide = (present >> s) >= 64;
		// arg-max of every sub-node (keys are distinct)
		if (wide && nsub < (uint32_t) nwarps) {
			// fewer sub-nodes than warps: each sub-node's keys are split over
			// W = nwarps / nsub warps, whose maxima meet in shared memory
			const uint32_t lw = ST_LOG_WARPS - s;  // log2 W
			const uint32_t W = 1u << lw, t = (uint32_t) warp >> lw, p = (uint32_t) warp & (W - 1u);
			const uint32_t ct = scnt[t], st = sstart[t];
			const uint32_t a = st + ((ct * p) >> lw), e = st + ((ct * (p + 1)) >> lw);
			uint64_t bk = 0;
			uint32_t bi = 0;
			for (uint32_t i = a + lane; i < e; i += 32)
				if (kc[i] > bk) {
					bk = kc[i];
					bi = i;
				}
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) {
				const uint64_t ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
				const uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
				if (ok > bk) {
					bk = ok;
					bi = oi;
				}
			}
			if (lane == 0) {
				s_pk[warp] = bk;
				s_pi[warp] = bi;
			}
			__syncthreads();
			if (threadIdx.x < nsub) {
				uint64_t mk = 0;
				uint32_t mi = 0;
				for (uint32_t q = threadIdx.x * W; q < threadIdx.x * W + W; q++)
					if (s_pk[q] > mk) {
						mk = s_pk[q];
						mi = s_pi[q];
					}
				topi[threadIdx.x] = (uint16_t) mi;
			}
		} else if (wide) {
			for (uint32_t t = warp; t < nsub; t += nwarps) {
				const uint32_t ct = scnt[t], st = sstart[t];
				uint64_t bk = 0;
				uint32_t bi = 0;
				for (uint32_t i = st + lane; i < st + ct; i += 32)
					if (kc[i] > bk) {
						bk = kc[i];
						bi = i;
					}
#pragma unroll
				for (int o = 16; o > 0; o >>= 1) {
					const uint64_t ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
					const uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
					if (ok > bk) {
						bk = ok;
						bi = oi;
					}
				}
				if (lane == 0)
					topi[t] = (uint16_t) bi;
			}
		} else {
			for (uint32_t t = threadIdx.x; t < nsub; t += ST_THREADS) {
				const uint32_t ct = scnt[t], st = sstart[t];
				uint64_t bk = 0;
				uint32_t bi = 0;
				for (uint32_t i = st; i < st + ct; i++)
					if (kc[i] > bk) {
						bk = kc[i];
						bi = i;
					}
				topi[t] = (uint16_t) bi;
			}
		}
		__syncthreads();
		// write the nodes of this sub-level (warps past the last sub-node skip whole)
		for (uint32_t tb = 0; tb < nsub; tb += ST_THREADS) {
			if (tb + (uint32_t) warp * 32 >= nsub)
				break;
			const uint32_t t = tb + threadIdx.x;
			bool occupied = false;
			uint32_t h = 0;
			if (t < nsub) {
				const uint32_t ct = scnt[t], st = sstart[t];
				h = (h0 << s) + t;
				if (ct > 0) {
					occupied = true;
					const uint32_t ti = topi[t];
					const Pt p = spts[sc[ti]];
					c.write_node(h, p);
					if (h < half) {
						T m = p.dim1;  // a node of one point: its own dim1
						if (ct >= 2) {
							uint32_t mi = st + ct / 2 - 1;
							if (ti <= mi)
								mi++;
							m = spts[sc[mi]].dim1;
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
		// drop each sub-node's point; every sub-node above the last level holds one.
		// Every key knows its sub-node t, so it moves on its own: past the t points
		// dropped before its sub-node, and its own sub-node's if that came first.  Of
		// the keys a sub-node keeps, the first floor(ct / 2) go to its left child.
		for (uint32_t i = threadIdx.x; i < present; i += ST_THREADS) {
			const uint32_t t = gc[i];
			const uint32_t ti = topi[t];
			if (i != ti) {
				const uint32_t ni = i - t - (i > ti ? 1u : 0u);
				const uint32_t rank = ni - (sstart[t] - t);  // among the sub-node's keys kept
				kn[ni] = kc[i];
				sn[ni] = sc[i];
				gn[ni] = (uint16_t) (2u * t + (rank >= (uint32_t) (scnt[t] >> 1) ? 1u : 0u));
			}
		}
		// spans of the next sub-level, in place: parents to registers, then children
		// (warps past the last sub-node have none)
		constexpr int PMAX = (ST_CAP / 2 + ST_THREADS - 1) / ST_THREADS;
		uint32_t pc[PMAX] = {}, ps[PMAX] = {};
		const bool spans = (uint32_t) warp * 32 < nsub;
		if (spans) {
#pragma unroll
			for (int u = 0; u < PMAX; u++) {
				const uint32_t t = threadIdx.x + u * ST_THREADS;
				if (t < nsub) {
					pc[u] = scnt[t];
					ps[u] = sstart[t];
				}
			}
		}
		__syncthreads();
		if (spans) {
#pragma unroll
			for (int u = 0; u < PMAX; u++) {
				const uint32_t t = threadIdx.x + u * ST_THREADS;
				if (t < nsub) {
					const uint32_t left = pc[u] / 2;
					scnt[2 * t] = (uint16_t) (pc[u] ? left : 0u);
					scnt[2 * t + 1] = (uint16_t) (pc[u] ? pc[u] - 1 - left : 0u);
					sstart[2 * t] = (uint16_t) (ps[u] - t);
					sstart[2 * t + 1] = (uint16_t) (ps[u] - t + left);
				}
			}
		}
		present -= nsub;
		uint64_t *tk = kc;
		kc = kn;
		kn = tk;
		uint16_t *ts = sc;
		sc = sn;
		sn = ts;
		ts = gc;
		gc = gn;
		gn = ts;
		__syncthreads();
	}

}

template <typename T>
T *as(void *p)
{
	return static_cast<T *>(p);
}

// All construction scratch lives in one device allocation (one cudaMalloc maps it
// far faster than a dozen stream-ordered allocations that regrow a trimmed pool).
struct ScratchLayout {
	size_t k1, kalt, c2, valt, k2, v32a, v32b, P, rs_status, rs_misc, hist1, flags, Ba, Bb, best, top, taken, tmax;
	size_t total;
};

ScratchLayout scratch_layout(pst_dtype dt, pst_idtype it, uint64_t n)
{
	ScratchLayout L{};
	const size_t ks = value_size(dt);
	const bool wide_key = dt == PST_F64;
	const uint32_t D = tree_levels(n);
	const uint32_t L0 = n ? std::min(subtree_level(n), D - 1) : 0;
	const uint64_t nodes_wide = 1ull << L0;
	const uint64_t rs_tiles = rs_num_tiles(n);
	const uint64_t ntiles = (n + TM_TILE - 1) / TM_TILE;
	size_t o = 0;
	auto take = [&](size_t bytes) {
		const size_t r = o;
		o = align_up(o + bytes);
		return r;
	};
	L.k1 = take(n * ks);
	L.kalt = take(n * ks);
	L.c2 = take(n * 8);
	L.valt = take(n * 8);
	L.k2 = take(wide_key ? n * 8 : 0);
	L.v32a = take(wide_key ? n * 4 : 0);
	L.v32b = take(wide_key ? n * 4 : 0);
	L.P = take(it == PST_ID_U32 ? n * 4 : 0);
	L.rs_status = take(256 * rs_tiles * 8);
	L.rs_misc = take(rs_misc_words() * 4);
	L.hist1 = take(RS_MAX_PASSES * 256 * 4);
	L.flags = take(256);
	L.Ba = take((nodes_wide + 1) * 4);
	L.Bb = take((nodes_wide + 1) * 4);
	L.best = take(nodes_wide * 8);
	L.top = take(nodes_wide * 4);
	L.taken = take(((n + 31) / 32) * 4);
	L.tmax = take(L0 ? ntiles * 8 : 0);
	L.total = o;
	return L;
}

struct Scratch {
	char *base = nullptr;
	explicit Scratch(size_t bytes)
	{
		cudaError_t e = cudaMalloc(&base, std::max<size_t>(bytes, 256));
		if (e == cudaErrorMemoryAllocation) {
			cudaGetLastError();
			fail(PST_ERR_NOMEM, "construction scratch allocation of " + std::to_string(bytes) + " B failed");
		}
		check_cuda(e, "cudaMalloc(construction scratch)");
	}
	~Scratch()
	{
		if (base)
			cudaFree(base);  // waits for the construction's work
	}
	Scratch(const Scratch &) = delete;
	Scratch &operator=(const Scratch &) = delete;
	template <typename T>
	T *at(size_t off) const
	{
		return reinterpret_cast<T *>(base + off);
	}
};

inline unsigned grid_for(uint64_t n, int threads)
{
	const uint64_t want = (n + threads - 1) / threads;
	const uint64_t cap = (uint64_t) device_info().sms * 16;
	return (unsigned) std::max<uint64_t>(1, std::min(want, cap));
}

// Scratch bytes of build_impl beyond the tree itself.
uint64_t build_scratch_bytes(pst_dtype dt, pst_idtype it, uint64_t n) { return scratch_layout(dt, it, n).total; }

// The tree's memory (one allocation; its occupancy bitmap cleared on `s`).  Called
// with the builder's sorts already queued on `s`: mapping several GB takes the host
// milliseconds, which then overlap the sorts instead of preceding them.
void alloc_tree(TreeStorage &t, cudaStream_t s)
{
	const TreeLayout L = tree_layout(t.dtype, t.idtype, t.n);
	cudaError_t e = cudaMalloc(&t.mem, L.total);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		t.mem = nullptr;
		fail(PST_ERR_NOMEM, "tree allocation of " + std::to_string(L.total) + " B failed");
	}
	check_cuda(e, "cudaMalloc(tree)");
	attach_tree_memory(t, t.mem);
	PST_CUDA(cudaMemsetAsync(t.occ, 0, L.total - L.off_occ, s));
}

template <typename T, bool HAS_ID>
void build_impl(TreeStorage &t, const void *pts_d, uint64_t n, cudaStream_t s)
{
	using K = typename KeyOf<T>::K;
	using Pt = Point<T, HAS_ID>;
	constexpr bool WIDE_KEY = sizeof(K) == 8;  // doubles: dim2 ranks from their own sort
	const Pt *pts = static_cast<const Pt *>(pts_d);
	const uint32_t D = t.levels;

	// ---- scratch
	const ScratchLayout SL = scratch_layout(t.dtype, t.idtype, n);
	Scratch scr(SL.total);
	void *k1 = scr.at<void>(SL.k1), *kalt = scr.at<void>(SL.kalt);
	uint64_t *c2 = scr.at<uint64_t>(SL.c2);
	void *valt = scr.at<void>(SL.valt);
	uint32_t *flag = scr.at<uint32_t>(SL.flags);  // [0] id order bits, [1] error bits, [2..3] id range, [4] -0.0 seen
	K *krange = reinterpret_cast<K *>(scr.at<unsigned char>(SL.flags) + 64);  // [k1 min, k1 max, k2 min, k2 max]
	{
		unsigned char init[256];
		memset(init, 0, sizeof(init));
		const uint32_t id_init[2] = {0xFFFFFFFFu, 0u};
		memcpy(init + 8, id_init, 8);
		const K kinit[4] = {~K(0), K(0), ~K(0), K(0)};
		memcpy(init + 64, kinit, sizeof(kinit));
		PST_CUDA(cudaMemcpyAsync(flag, init, sizeof(init), cudaMemcpyHostToDevice, s));
	}
	// one SortScratch for every sort of this build: its epoch tags the look-back
	// status of each pass, which is cleared only here
	SortScratch sc;
	sc.status = scr.at<uint64_t>(SL.rs_status);
	sc.hist = scr.at<uint32_t>(SL.rs_misc);
	sc.counters = sc.hist + RS_MAX_PASSES * 256;
	sc.err = flag + 1;
	PST_CUDA(cudaMemsetAsync(sc.status, 0, 256 * rs_num_tiles(n) * 8, s));

	const unsigned g = grid_for(n, 256);
	// ---- keys, made in input order; the same pass checks the ids and counts the
	// dim1 keys' digits for their sort
	uint32_t *hist1 = scr.at<uint32_t>(SL.hist1);
	PST_CUDA(cudaMemsetAsync(hist1, 0, RS_MAX_PASSES * 256 * 4, s));
	const size_t pk_smem = (size_t) PK_HIST_COPIES * sizeof(K) * 256 * 4;
	k_prep_keys<T, HAS_ID, HAS_ID><<<g, 256, pk_smem, s>>>(pts, nullptr, n, static_cast<K *>(k1), c2,
	                                                       scr.at<K>(SL.k2), krange, flag + 4, flag, flag + 2,
	                                                       hist1);
	PST_CUDA(cudaGetLastError());
	K range[4];
	uint32_t negzero = 0, idscan[4] = {0, 0, 0, 0};
	PST_CUDA(cudaMemcpyAsync(range, krange, sizeof(range), cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaMemcpyAsync(&negzero, flag + 4, 4, cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaMemcpyAsync(idscan, flag, 16, cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaStreamSynchronize(s));
	// ---- tiebreak order (id, input index): the input order unless the ids decrease
	// somewhere, then the keys are made again in the order of one sort of the ids
	const uint32_t *P = nullptr;
	bool ids_are_indices = true;
	if constexpr (HAS_ID) {
		ids_are_indices = !(idscan[0] & 2u);
		if (idscan[0] & 1u) {
			uint32_t *idk = static_cast<uint32_t *>(k1);  // k1 holds at least n u32
			k_id_keys<T, HAS_ID><<<g, 256, 0, s>>>(pts, n, idk);
			sc.keys_alt = kalt;
			sc.vals_alt = valt;  // n u32 fit in the u64 buffers
			sc.vals_tmp = c2;
			uint32_t *kres, *vres;
			radix_sort<uint32_t, uint32_t>(idk, nullptr, n, rs_passes<uint32_t>(idscan[2], idscan[3]), sc, &kres,
			                               &vres, s);
			// ids decrease somewhere, so they are not all equal and the sort ran
			PST_CUDA(cudaMemcpyAsync(scr.at<uint32_t>(SL.P), vres, n * 4, cudaMemcpyDeviceToDevice, s));
			P = scr.at<uint32_t>(SL.P);
			// the same keys in the new order: ranges and digit counts stand, so neither
			// is made again (the sort's error bits in flag[1] are kept)
			k_prep_keys<T, HAS_ID, false><<<g, 256, 0, s>>>(pts, P, n, static_cast<K *>(k1), c2, scr.at<K>(SL.k2),
			                                                krange, flag + 4, nullptr, nullptr, nullptr);
			PST_CUDA(cudaGetLastError());
		}
	}
	if constexpr (WIDE_KEY) {
		// dim2 ranks: stable sort of the dim2 keys in tiebreak order
		sc.keys_alt = kalt;
		sc.vals_alt = scr.at<void>(SL.v32a);
		sc.vals_tmp = scr.at<void>(SL.v32b);
		K *kres;
		uint32_t *S2;
		radix_sort<K, uint32_t>(scr.at<K>(SL.k2), nullptr, n, rs_passes<K>(range[2], range[3]), sc, &kres, &S2, s);
		k_rank_keys<<<g, 256, 0, s>>>(S2, n, c2);
		PST_CUDA(cudaGetLastError());
	}
	// ---- dim1 order, carrying the dim2 keys
	K *k1s;
	uint64_t *c2s;
	{
		sc.keys_alt = kalt;
		sc.vals_alt = valt;
		sc.vals_tmp = nullptr;
		radix_sort<K, uint64_t>(static_cast<K *>(k1), c2, n, rs_passes<K>(range[0], range[1]), sc, &k1s, &c2s, s,
		                        hist1);
	}
	alloc_tree(t, s);

	// ---- levels
	const uint32_t L0 = std::min(subtree_level(n), D - 1);
	const uint64_t nodes_wide = 1ull << L0;
	const uint64_t ntiles = (n + TM_TILE - 1) / TM_TILE;
	unsigned long long *best = scr.at<unsigned long long>(SL.best);
	PST_CUDA(cudaMemsetAsync(scr.at<void>(SL.taken), 0, ((n + 31) / 32) * 4, s));
	BuildCtx<T, HAS_ID> c;
	c.pts = pts;
	c.P = P;
	// points rebuilt from the keys: 4-byte values, no -0.0, ids (if any) = input indices
	c.recon = !WIDE_KEY && !negzero && ids_are_indices && P == nullptr;
	c.k1s = k1s;
	c.c2s = c2s;
	c.taken = scr.at<uint32_t>(SL.taken);
	c.tmax = scr.at<uint64_t>(SL.tmax);
	c.dim1 = as<T>(t.dim1);
	c.dim2 = as<T>(t.dim2);
	c.med = as<T>(t.med);
	c.id = t.id;
	c.occ = t.occ;
	c.top_pos = scr.at<uint32_t>(SL.top);
	c.err = flag + 1;
	c.n = n;
	c.D = D;
	uint32_t *B = scr.at<uint32_t>(SL.Ba), *Bn = scr.at<uint32_t>(SL.Bb);
	{
		const uint32_t b0[2] = {0u, (uint32_t) n};
		PST_CUDA(cudaMemcpyAsync(B, b0, 8, cudaMemcpyHostToDevice, s));
	}
	if (L0) {
		const unsigned tgrid = (unsigned) std::max<uint64_t>(
		    1, std::min<uint64_t>((ntiles + AM_THREADS / 32 - 1) / (AM_THREADS / 32), (uint64_t) device_info().sms * 8));
		k_tile_max_all<<<tgrid, AM_THREADS, 0, s>>>(c2s, c.taken, n, c.tmax);
		const unsigned am_grid = (unsigned) std::max<uint64_t>(
		    1, std::min<uint64_t>((ntiles + AM_THREADS - 1) / AM_THREADS, (uint64_t) device_info().sms * 8));
		for (uint32_t d = 0; d < L0; d++) {
			const uint32_t nseg = 1u << d;
			PST_CUDA(cudaMemsetAsync(best, 0, (size_t) nseg * 8, s));
			k_level_argmax<<<am_grid, AM_THREADS, 0, s>>>(c2s, c.taken, c.tmax, n, B, nseg, best, c.err,
			                                               (float) ((double) nseg / (double) n));
			k_level_nodes<T, HAS_ID><<<(nseg + 127) / 128, 128, 0, s>>>(c, d, B, Bn, best);
			if (d + 1 < L0)
				k_tile_refresh<<<(unsigned) ((nseg * 32 + AM_THREADS - 1) / AM_THREADS), AM_THREADS, 0, s>>>(
				    c2s, c.taken, n, c.top_pos, d, c.tmax, c.err);
			PST_CUDA(cudaGetLastError());
			std::swap(B, Bn);
		}
	}
	constexpr size_t st_bytes = SubtreeSmem<T, HAS_ID>::BYTES;
	PST_CUDA(cudaFuncSetAttribute(k_subtree<T, HAS_ID>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) st_bytes));
	k_subtree<T, HAS_ID><<<(unsigned) nodes_wide, ST_THREADS, st_bytes, s>>>(c, L0, B);
	PST_CUDA(cudaGetLastError());
	uint32_t errs[2] = {0, 0};
	PST_CUDA(cudaMemcpyAsync(errs, flag, 8, cudaMemcpyDeviceToHost, s));
	PST_CUDA(cudaStreamSynchronize(s));
	if (errs[1])
		fail(PST_ERR_INTERNAL, "construction consistency check failed (code " + std::to_string(errs[1]) + ")");
}

}  // namespace

uint64_t tree_bytes(pst_dtype dt, pst_idtype it, uint64_t n) { return tree_layout(dt, it, n).total; }

void attach_tree_memory(TreeStorage &t, void *mem)
{
	const TreeLayout L = tree_layout(t.dtype, t.idtype, t.n);
	t.mem = mem;
	t.bytes = L.total;
	char *b = static_cast<char *>(mem);
	t.dim1 = b + L.off_dim1;
	t.dim2 = b + L.off_dim2;
	t.med = b + L.off_med;
	t.id = t.idtype == PST_ID_U32 ? reinterpret_cast<uint32_t *>(b + L.off_id) : nullptr;
	t.occ = reinterpret_cast<uint32_t *>(b + L.off_occ);
}

// The separately allocated search indexes of finish_tree_aux.
static uint64_t aux_bytes(pst_dtype dt, uint64_t n)
{
	const uint32_t D = tree_levels(n);
	if (D < 8)
		return 0;
	const uint64_t last_par = ((1ull << (D - 2)) / 64 + 31) / 32 * 4;
	return last_par + (1ull << (D - 1)) / 64 * value_size(dt);
}

uint64_t build_bytes_needed(pst_dtype dt, pst_idtype it, uint64_t n)
{
	return tree_bytes(dt, it, n) + build_scratch_bytes(dt, it, n) + aux_bytes(dt, n);
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
	try {
		// the tree's own memory is allocated by build_impl once its sorts are queued
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
		finish_tree_aux(t, s);
		PST_CUDA(cudaStreamSynchronize(s));
	} catch (...) {
		cudaStreamSynchronize(s);
		free_tree(t);
		throw;
	}
}

namespace {

// Block j of level L: positions [2^L + 64 j, 2^L + 64 j + 64); its children are the
// 128 positions from 2^(L+1) + 128 j, i.e. occupancy words 2^(L+1)/32 + 4 j .. + 3.
__global__ void k_last_par(const uint32_t *__restrict__ occ, uint32_t L, uint32_t *out)
{
	const uint64_t nb = (1ull << L) / 64;
	const uint64_t w0 = (1ull << (L + 1)) / 32;
	for (uint64_t j = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; j < ((nb + 31) & ~31ull);
	     j += (uint64_t) gridDim.x * blockDim.x) {
		bool any = false;
		if (j < nb) {
			const uint4 o = *reinterpret_cast<const uint4 *>(occ + w0 + 4 * j);
			any = (o.x | o.y | o.z | o.w) != 0;
		}
		const uint32_t bits = __ballot_sync(0xFFFFFFFFu, any);
		if ((threadIdx.x & 31) == 0)
			out[j >> 5] = bits;
	}
}

// Minimum of two dim2 values that keeps a NaN (so that no query's min2 compares
// at most the minimum of a block with a NaN below it).
template <typename T>
__device__ __forceinline__ T min_keep_nan(T a, T b)
{
	if constexpr (std::is_floating_point<T>::value) {
		if (a != a)
			return a;
		if (b != b)
			return b;
	}
	return b < a ? b : a;
}

// sub_min of the 64-slot blocks of level e (one warp per block): its 128 children
// on level e + 1 (positions 2^(e+1) + 128 j ..), only the occupied ones when that
// is the last level, and the sub_min of the two child blocks below them.
template <typename T>
__global__ void k_sub_min(const T *__restrict__ dim2, const uint32_t *__restrict__ occ, T *sub_min, uint32_t D,
                          uint32_t e)
{
	const uint64_t nb = (1ull << e) / 64;
	const uint32_t lane = threadIdx.x & 31;
	for (uint64_t j = ((uint64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nb;
	     j += ((uint64_t) gridDim.x * blockDim.x) >> 5) {
		const uint64_t c0 = (1ull << (e + 1)) + 128 * j;  // first child position
		const uint64_t p = c0 + 4 * lane;
		T v[4];
		if constexpr (sizeof(T) == 4) {
			const uint4 x = *reinterpret_cast<const uint4 *>(dim2 + p);
			memcpy(&v[0], &x.x, 4);
			memcpy(&v[1], &x.y, 4);
			memcpy(&v[2], &x.z, 4);
			memcpy(&v[3], &x.w, 4);
		} else {
			const double2 a = reinterpret_cast<const double2 *>(dim2 + p)[0];
			const double2 b = reinterpret_cast<const double2 *>(dim2 + p)[1];
			v[0] = a.x;
			v[1] = a.y;
			v[2] = b.x;
			v[3] = b.y;
		}
		// children on the last level exist where their occupancy bit is set
		const uint32_t om = e + 2 == D ? (occ[p >> 5] >> (p & 31)) & 0xFu : 0xFu;
		bool have = false;
		T m = T(0);
#pragma unroll
		for (int k = 0; k < 4; k++)
			if ((om >> k) & 1u) {
				m = have ? min_keep_nan(m, v[k]) : v[k];
				have = true;
			}
		if (lane == 0 && e + 2 < D) {
			// the child blocks' own descendants (levels e + 2 .. D - 1)
			const T a = sub_min[c0 >> 6], b = sub_min[(c0 >> 6) + 1];
			m = have ? min_keep_nan(min_keep_nan(m, a), b) : min_keep_nan(a, b);
			have = true;
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			const T om2 = __shfl_xor_sync(0xFFFFFFFFu, m, o);
			const bool oh = __shfl_xor_sync(0xFFFFFFFFu, have, o);
			if (oh)
				m = have ? min_keep_nan(m, om2) : om2;
			have = have || oh;
		}
		if (lane == 0) {
			// a block without descendants holds nothing to test: the largest value
			T none;
			if constexpr (std::is_floating_point<T>::value)
				none = std::numeric_limits<T>::infinity();
			else
				none = std::numeric_limits<T>::max();
			sub_min[((1ull << e) >> 6) + j] = have ? m : none;
		}
	}
}

}  // namespace

void finish_tree_aux(TreeStorage &t, cudaStream_t s)
{
	if (t.levels < 8)  // level D-2 spans less than one 64-slot block
		return;
	const uint32_t L = t.levels - 2;
	const uint64_t nb = (1ull << L) / 64;
	const uint64_t words = (nb + 31) / 32;
	cudaError_t e = cudaMalloc(&t.last_par, words * 4);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		fail(PST_ERR_NOMEM, "search index allocation failed");
	}
	check_cuda(e, "cudaMalloc(search index)");
	const unsigned g = (unsigned) std::max<uint64_t>(1, std::min<uint64_t>((nb + 255) / 256, 65535));
	k_last_par<<<g, 256, 0, s>>>(t.occ, L, t.last_par);
	PST_CUDA(cudaGetLastError());
	// sub_min: one value per 64-slot block of positions [64, 2^(D-1)), levels
	// 6..D-2, built from the bottom up
	const size_t vs = value_size(t.dtype);
	e = cudaMalloc(&t.sub_min, ((1ull << (t.levels - 1)) / 64) * vs);
	if (e == cudaErrorMemoryAllocation) {
		cudaGetLastError();
		fail(PST_ERR_NOMEM, "search index allocation failed");
	}
	check_cuda(e, "cudaMalloc(search index)");
	for (uint32_t lv = t.levels - 2; lv >= 6; lv--) {
		const uint64_t warps = (1ull << lv) / 64;
		const unsigned gb = (unsigned) std::max<uint64_t>(1, std::min<uint64_t>((warps * 32 + 255) / 256, 1u << 20));
		switch (t.dtype) {
		case PST_F32:
			k_sub_min<float><<<gb, 256, 0, s>>>(static_cast<const float *>(t.dim2), t.occ,
			                                    static_cast<float *>(t.sub_min), t.levels, lv);
			break;
		case PST_F64:
			k_sub_min<double><<<gb, 256, 0, s>>>(static_cast<const double *>(t.dim2), t.occ,
			                                     static_cast<double *>(t.sub_min), t.levels, lv);
			break;
		case PST_I32:
			k_sub_min<int32_t><<<gb, 256, 0, s>>>(static_cast<const int32_t *>(t.dim2), t.occ,
			                                      static_cast<int32_t *>(t.sub_min), t.levels, lv);
			break;
		}
		PST_CUDA(cudaGetLastError());
	}
}

void free_tree(TreeStorage &t)
{
	if (t.mem)
		cudaFree(t.mem);
	t.mem = nullptr;
	if (t.last_par)
		cudaFree(t.last_par);
	t.last_par = nullptr;
	if (t.sub_min)
		cudaFree(t.sub_min);
	t.sub_min = nullptr;
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
