// Device-wide exclusive scan and a stable LSD radix sort (unsigned keys with a
// uint32 payload), written for the construction path.  The reference sorts
// size_t index arrays with thrust::sort and an indirect comparator
// (pst/static-pst-gpu.tu:248-318); here the comparator is folded into an
// order-preserving key and the sort moves 4- or 8-byte keys plus 4-byte payloads.
#pragma once

#include <algorithm>

#include "common.cuh"

namespace pst {

// ---------------------------------------------------------------------------
// Exclusive scan (three kernels: tile reduce, scan of tile sums, tile scan).

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__device__ T block_excl_scan(T v, T *total, T *warp_sums)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
	T inc = warp_incl_scan(v);
	if (lane == 31)
		warp_sums[warp] = inc;
	__syncthreads();
	if (warp == 0) {
		T s = lane < nw ? warp_sums[lane] : T(0);
		T si = warp_incl_scan(s);
		if (lane < nw)
			warp_sums[lane] = si - s;
		if (lane == nw - 1)
			warp_sums[32] = si;
	}
	__syncthreads();
	T r = warp_sums[warp] + inc - v;
	*total = warp_sums[32];
	__syncthreads();
	return r;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const T *in, uint64_t n, T *tile_sums)
{
	__shared__ T ws[33];
	const uint64_t base = (uint64_t) blockIdx.x * SCAN_TILE + (uint64_t) threadIdx.x * SCAN_ITEMS;
	T s = 0;
#pragma unroll
	for (int i = 0; i < SCAN_ITEMS; i++)
		if (base + i < n)
			s += in[base + i];
	T tot;
	block_excl_scan(s, &tot, ws);
	if (threadIdx.x == 0)
		tile_sums[blockIdx.x] = tot;
}

// One block scans `n` tile sums in place (exclusive), writing the grand total.
template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(T *sums, uint64_t n, T *total_out)
{
	__shared__ T ws[33];
	T carry = 0;
	for (uint64_t c0 = 0; c0 < n; c0 += SCAN_TILE) {
		const uint64_t base = c0 + (uint64_t) threadIdx.x * SCAN_ITEMS;
		T v[SCAN_ITEMS];
		T s = 0;
#pragma unroll
		for (int i = 0; i < SCAN_ITEMS; i++) {
			v[i] = base + i < n ? sums[base + i] : T(0);
			s += v[i];
		}
		T tot;
		T ex = block_excl_scan(s, &tot, ws) + carry;
#pragma unroll
		for (int i = 0; i < SCAN_ITEMS; i++) {
			if (base + i < n)
				sums[base + i] = ex;
			ex += v[i];
		}
		carry += tot;
	}
	if (threadIdx.x == 0 && total_out)
		*total_out = carry;
}

template <typename T, typename U>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const T *in, U *out, uint64_t n, const T *tile_offs)
{
	__shared__ T ws[33];
	const uint64_t base = (uint64_t) blockIdx.x * SCAN_TILE + (uint64_t) threadIdx.x * SCAN_ITEMS;
	T v[SCAN_ITEMS];
	T s = 0;
#pragma unroll
	for (int i = 0; i < SCAN_ITEMS; i++) {
		v[i] = base + i < n ? in[base + i] : T(0);
		s += v[i];
	}
	T tot;
	T ex = block_excl_scan(s, &tot, ws) + tile_offs[blockIdx.x];
#pragma unroll
	for (int i = 0; i < SCAN_ITEMS; i++) {
		if (base + i < n)
			out[base + i] = (U) ex;
		ex += v[i];
	}
}

// Exclusive scan of n values (in may equal out).  `tmp` needs scan_tmp_elems(n)
// entries of T; the grand total goes to total_d when non-null.
inline uint64_t scan_tmp_elems(uint64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

template <typename T, typename U = T>
void exclusive_scan(const T *in, U *out, uint64_t n, T *tmp, T *total_d, cudaStream_t s)
{
	if (n == 0) {
		if (total_d)
			PST_CUDA(cudaMemsetAsync(total_d, 0, sizeof(T), s));
		return;
	}
	const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
	k_scan_reduce<T><<<(unsigned) tiles, SCAN_THREADS, 0, s>>>(in, n, tmp);
	k_scan_tiles<T><<<1, SCAN_THREADS, 0, s>>>(tmp, tiles, total_d);
	k_scan_apply<T, U><<<(unsigned) tiles, SCAN_THREADS, 0, s>>>(in, out, n, tmp);
	PST_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// LSD radix sort, 8-bit digits, 4096-key tiles.  Stable: within a tile keys are
// ranked in input order (warp-private digit counters; the lanes of a warp holding
// the same digit are found with eight ballots, one per digit bit), and tiles take
// their digit offsets from a digit-major exclusive scan.  Only the passes that
// cover bits where the keys differ are run: keys between kmin and kmax share
// every bit above the highest bit of kmin ^ kmax.

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;
static_assert(RS_THREADS == 256, "one thread per digit in the digit scans");

template <typename K>
__device__ __forceinline__ uint32_t rs_digit(K k, int shift) { return (uint32_t) (k >> shift) & 0xFFu; }

// Mask of the valid lanes of this warp that hold the same digit as this lane.
__device__ __forceinline__ uint32_t rs_peers(uint32_t d, bool valid)
{
	uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
	for (int b = 0; b < 8; b++) {
		const bool bit = (d >> b) & 1u;
		const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
		peers &= bit ? m : ~m;
	}
	return peers;
}

// Per-tile digit counts, digit-major: tile_hist[digit * num_tiles + tile].
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const K *keys, uint64_t n, int shift, uint32_t *tile_hist,
                                                           uint32_t num_tiles)
{
	__shared__ uint32_t h[RS_WARPS][256];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS)
		(&h[0][0])[i] = 0;
	__syncthreads();
	const uint64_t t0 = (uint64_t) blockIdx.x * RS_TILE;
#pragma unroll 4
	for (int i = 0; i < RS_ITEMS; i++) {
		const uint64_t idx = t0 + (uint64_t) warp * (RS_ITEMS * 32) + i * 32 + lane;
		if (idx < n)
			atomicAdd(&h[warp][rs_digit(keys[idx], shift)], 1u);
	}
	__syncthreads();
	uint32_t s = 0;
#pragma unroll
	for (int w = 0; w < RS_WARPS; w++)
		s += h[w][threadIdx.x];
	tile_hist[(uint64_t) threadIdx.x * num_tiles + blockIdx.x] = s;
}

// One pass.  vals_in == nullptr means the identity payload (the key's input index;
// 32-bit payloads only).
template <typename K, typename V>
__global__ void __launch_bounds__(RS_THREADS) k_rs_downsweep(const K *keys_in, const V *vals_in, K *keys_out,
                                                             V *vals_out, uint64_t n, int shift,
                                                             const uint32_t *tile_off, uint32_t num_tiles)
{
	extern __shared__ __align__(16) unsigned char rs_smem[];
	V *sv = reinterpret_cast<V *>(rs_smem);
	K *sk = reinterpret_cast<K *>(sv + RS_TILE);
	uint32_t *whist = reinterpret_cast<uint32_t *>(sk + RS_TILE);  // [RS_WARPS][256]
	uint32_t *dstart = whist + RS_WARPS * 256;                      // [256] tile-local digit start
	uint32_t *gbase = dstart + 256;                                 // [256] global start of the digit for this tile
	uint32_t *wsum = gbase + 256;                                   // [33]

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS)
		whist[i] = 0;
	gbase[threadIdx.x] = tile_off[(uint64_t) threadIdx.x * num_tiles + blockIdx.x];
	__syncthreads();

	const uint64_t t0 = (uint64_t) blockIdx.x * RS_TILE;
	K k[RS_ITEMS];
	V v[RS_ITEMS];
	uint32_t loc[RS_ITEMS];
#pragma unroll
	for (int i = 0; i < RS_ITEMS; i++) {
		const uint64_t idx = t0 + (uint64_t) warp * (RS_ITEMS * 32) + i * 32 + lane;
		const bool valid = idx < n;
		k[i] = valid ? keys_in[idx] : K(0);
		v[i] = valid ? (vals_in ? vals_in[idx] : (V) idx) : V(0);
		const uint32_t d = rs_digit(k[i], shift);
		const uint32_t peers = rs_peers(d, valid);
		const int leader = valid ? __ffs(peers) - 1 : lane;
		uint32_t old = 0;
		if (valid && lane == leader) {
			old = whist[warp * 256 + d];
			whist[warp * 256 + d] = old + __popc(peers);
		}
		old = __shfl_sync(0xFFFFFFFFu, old, leader);
		loc[i] = old + __popc(peers & lanemask_lt());
		__syncwarp();  // the next item's leaders read the counters written here
	}
	__syncthreads();
	// Exclusive prefix of each digit over warps, then over digits.
	{
		const int d = threadIdx.x;
		uint32_t run = 0;
#pragma unroll
		for (int w = 0; w < RS_WARPS; w++) {
			uint32_t t = whist[w * 256 + d];
			whist[w * 256 + d] = run;
			run += t;
		}
		uint32_t tot;
		dstart[d] = block_excl_scan<uint32_t>(run, &tot, wsum);
	}
	__syncthreads();
#pragma unroll
	for (int i = 0; i < RS_ITEMS; i++) {
		const uint64_t idx = t0 + (uint64_t) warp * (RS_ITEMS * 32) + i * 32 + lane;
		if (idx < n) {
			const uint32_t d = rs_digit(k[i], shift);
			const uint32_t lp = dstart[d] + whist[warp * 256 + d] + loc[i];
			sk[lp] = k[i];
			sv[lp] = v[i];
		}
	}
	__syncthreads();
	const uint64_t rem_n = n - t0;
	const uint32_t tile_n = rem_n < (uint64_t) RS_TILE ? (uint32_t) rem_n : (uint32_t) RS_TILE;
	for (uint32_t j = threadIdx.x; j < tile_n; j += RS_THREADS) {
		const K key = sk[j];
		const uint32_t d = rs_digit(key, shift);
		const uint64_t g = (uint64_t) gbase[d] + (j - dstart[d]);
		keys_out[g] = key;
		vals_out[g] = sv[j];
	}
}

template <typename K, typename V>
constexpr size_t rs_downsweep_smem()
{
	return RS_TILE * (sizeof(K) + sizeof(V)) + (RS_WARPS * 256 + 256 + 256 + 33) * 4;
}

inline uint64_t rs_num_tiles(uint64_t n) { return (n + RS_TILE - 1) / RS_TILE; }

// Scratch for radix_sort: key/value ping-pong buffers of n entries plus the tile
// histogram and its scan temporaries.
struct SortScratch {
	void *keys_alt = nullptr;  // n keys
	void *vals_alt = nullptr;  // n payloads
	void *vals_tmp = nullptr;  // n payloads (second buffer for an identity input payload)
	uint32_t *tile_hist = nullptr;
	uint32_t *scan_tmp = nullptr;
};

// Number of 8-bit passes needed to sort keys lying in [kmin, kmax].
template <typename K>
inline int rs_passes(K kmin, K kmax)
{
	const uint64_t diff = (uint64_t) (kmin ^ kmax);
	if (!diff)
		return 0;
	int bits = 64 - __builtin_clzll(diff);
	return (bits + 7) / 8;
}

// Sorts (keys, vals) ascending by key, stably, over the first `passes` digits.
// vals may be null (identity payload, 32-bit payloads only).  The sorted data is in
// the buffers returned through *keys_res / *vals_res (the input buffers or the
// scratch ones; *vals_res stays null when passes == 0 and vals is null).
template <typename K, typename V>
void radix_sort(K *keys, V *vals, uint64_t n, int passes, SortScratch &sc, K **keys_res, V **vals_res, cudaStream_t s)
{
	*keys_res = keys;
	*vals_res = vals;
	if (n == 0 || passes == 0)
		return;
	const uint64_t tiles = rs_num_tiles(n);
	PST_CUDA(cudaFuncSetAttribute(k_rs_downsweep<K, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                              (int) rs_downsweep_smem<K, V>()));
	K *kin = keys, *kout = static_cast<K *>(sc.keys_alt);
	V *vin = vals;
	V *vout = static_cast<V *>(sc.vals_alt);
	for (int p = 0; p < passes; p++) {
		k_rs_upsweep<K><<<(unsigned) tiles, RS_THREADS, 0, s>>>(kin, n, 8 * p, sc.tile_hist, (uint32_t) tiles);
		exclusive_scan<uint32_t>(sc.tile_hist, sc.tile_hist, 256 * tiles, sc.scan_tmp, nullptr, s);
		k_rs_downsweep<K, V><<<(unsigned) tiles, RS_THREADS, rs_downsweep_smem<K, V>(), s>>>(
		    kin, vin, kout, vout, n, 8 * p, sc.tile_hist, (uint32_t) tiles);
		PST_CUDA(cudaGetLastError());
		K *kt = kin;
		kin = kout;
		kout = kt;
		V *vt = vin;
		vin = vout;
		vout = vt ? vt : static_cast<V *>(sc.vals_tmp);
	}
	*keys_res = kin;
	*vals_res = vin;
}

}  // namespace pst
