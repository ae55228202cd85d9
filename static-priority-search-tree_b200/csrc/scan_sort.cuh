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
// LSD radix sort, 8-bit digits, 4096-key tiles, one kernel per digit pass: the
// single-pass scheme of Adinets and Merrill, "Onesweep: A Faster Least Significant
// Digit Radix Sort for GPUs" (2022), written for this library.  A first kernel
// histograms the digits of every pass at once; in a
// pass, each tile ranks its keys stably (warp-private digit counters; the lanes of
// a warp holding the same digit are found with eight ballots, one per digit bit),
// publishes its digit counts, and finds the counts of all earlier tiles by walking
// back over their published aggregates until one carries an inclusive prefix
// (decoupled look-back).  Tiles take their numbers from an atomic counter in the
// order they start, so a tile only waits on tiles that are already running; every
// wait is bounded and a wait that runs out raises an error flag instead of
// scattering.  Keys move once per pass: read, staged in shared memory in sorted
// order, written with coalesced runs.  Only the passes that cover bits where the
// keys differ are run: keys between kmin and kmax share every bit above the
// highest bit of kmin ^ kmax.

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_MAX_PASSES = 8;
static_assert(RS_THREADS == 256, "one thread per digit in the digit scans");

// Look-back status word of (tile, digit): flag (2 bits) | epoch (30 bits) | count.
constexpr uint64_t RS_AGG = 1ull << 62, RS_PREFIX = 2ull << 62, RS_FLAGS = 3ull << 62;
constexpr uint32_t RS_SPIN_LIMIT = 1u << 22;
constexpr uint32_t RS_ERR_LOOKBACK = 32u;  // error bit raised when a look-back wait runs out

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

// hist[p * 256 + digit] += count of keys with that digit in pass p, for p < passes.
// Warps of a block pair up on private shared-memory histograms.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_global_hist(const K *__restrict__ keys, uint64_t n, int passes,
                                                               uint32_t *hist)
{
	constexpr int COPIES = 4;
	extern __shared__ uint32_t gh_smem[];  // [COPIES][passes * 256]
	const int words = passes * 256;
	for (int i = threadIdx.x; i < COPIES * words; i += RS_THREADS)
		gh_smem[i] = 0;
	__syncthreads();
	uint32_t *h = gh_smem + ((threadIdx.x >> 5) % COPIES) * words;
	constexpr int IT = 8;  // loads issued before their atomics
	const uint64_t step = (uint64_t) gridDim.x * blockDim.x * IT;
	for (uint64_t base = (uint64_t) blockIdx.x * blockDim.x * IT + threadIdx.x; base < n; base += step) {
		K k[IT];
#pragma unroll
		for (int u = 0; u < IT; u++) {
			const uint64_t i = base + (uint64_t) u * blockDim.x;
			k[u] = i < n ? keys[i] : K(0);
		}
#pragma unroll
		for (int u = 0; u < IT; u++) {
			if (base + (uint64_t) u * blockDim.x < n)
				for (int p = 0; p < passes; p++)
					atomicAdd(&h[p * 256 + rs_digit(k[u], 8 * p)], 1u);
		}
	}
	__syncthreads();
	for (int i = threadIdx.x; i < words; i += RS_THREADS) {
		uint32_t t = 0;
#pragma unroll
		for (int c = 0; c < COPIES; c++)
			t += gh_smem[c * words + i];
		if (t)
			atomicAdd(&hist[i], t);
	}
}

// One pass.  vals_in == nullptr means the identity payload (the key's input index;
// 32-bit payloads only).  The tile's payloads are copied into shared memory
// asynchronously as soon as the tile is known, so their reads overlap the ranking
// and the look-back; each sorted key carries its input slot to find its payload.
template <typename K, typename V>
__global__ void __launch_bounds__(RS_THREADS, 3) k_rs_onesweep(const K *keys_in, const V *vals_in, K *keys_out,
                                                            V *vals_out, uint64_t n, int shift,
                                                            const uint32_t *__restrict__ hist, uint64_t *status,
                                                            uint32_t *tile_counter, uint32_t epoch, uint32_t *err)
{
	extern __shared__ __align__(16) unsigned char rs_smem[];
	V *sv = reinterpret_cast<V *>(rs_smem);                         // payloads, input order
	K *sk = reinterpret_cast<K *>(sv + RS_TILE);                    // keys, sorted within the tile
	uint16_t *si = reinterpret_cast<uint16_t *>(sk + RS_TILE);      // input slot of each sorted key
	uint32_t *whist = reinterpret_cast<uint32_t *>(si + RS_TILE);   // [RS_WARPS][256]
	uint32_t *dstart = whist + RS_WARPS * 256;                      // [256] tile-local digit start
	uint32_t *gbase = dstart + 256;                                 // [256] global start of the digit for this tile
	uint32_t *wsum = gbase + 256;                                   // [33]
	__shared__ uint32_t s_tile, s_fail;

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (threadIdx.x == 0) {
		s_tile = atomicAdd(tile_counter, 1u);
		s_fail = 0;
	}
	for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS)
		whist[i] = 0;
	__syncthreads();
	const uint32_t tile = s_tile;
	const uint64_t t0 = (uint64_t) tile * RS_TILE;
	const uint64_t rem_n = n - t0;
	const uint32_t tile_n = rem_n < (uint64_t) RS_TILE ? (uint32_t) rem_n : (uint32_t) RS_TILE;
	if (vals_in) {
		// 16-byte copies, then the (4-byte multiple) tail of a partial last tile
		const unsigned char *src = reinterpret_cast<const unsigned char *>(vals_in + t0);
		unsigned char *dst = reinterpret_cast<unsigned char *>(sv);
		const uint32_t bytes = tile_n * (uint32_t) sizeof(V), body = bytes & ~15u;
		for (uint32_t o = threadIdx.x * 16u; o < body; o += RS_THREADS * 16u)
			cp_async16(dst + o, src + o);
		for (uint32_t o = body + threadIdx.x * 4u; o < bytes; o += RS_THREADS * 4u)
			cp_async4(dst + o, src + o);
		cp_async_commit();
	}
	K k[RS_ITEMS];
	uint32_t loc[RS_ITEMS];
#pragma unroll
	for (int i = 0; i < RS_ITEMS; i++) {
		const uint64_t idx = t0 + (uint64_t) warp * (RS_ITEMS * 32) + i * 32 + lane;
		k[i] = idx < n ? keys_in[idx] : K(0);
	}
#pragma unroll
	for (int i = 0; i < RS_ITEMS; i++) {
		const uint64_t idx = t0 + (uint64_t) warp * (RS_ITEMS * 32) + i * 32 + lane;
		const bool valid = idx < n;
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
	{
		const uint32_t d = threadIdx.x;
		uint32_t cnt = 0;
#pragma unroll
		for (int w = 0; w < RS_WARPS; w++) {
			const uint32_t t = whist[w * 256 + d];
			whist[w * 256 + d] = cnt;
			cnt += t;
		}
		// publish this tile's count, then gather the counts of the tiles before it
		volatile uint64_t *st = reinterpret_cast<volatile uint64_t *>(status);
		const uint64_t tag = (uint64_t) (epoch & 0x3FFFFFFFu) << 32;
		uint64_t excl = 0;
		if (tile == 0) {
			st[d] = RS_PREFIX | tag | cnt;
		} else {
			st[(uint64_t) tile * 256 + d] = RS_AGG | tag | cnt;
			int64_t t = (int64_t) tile - 1;
			uint32_t spins = 0;
			for (;;) {
				const uint64_t x = st[(uint64_t) t * 256 + d];
				const uint64_t f = x & RS_FLAGS;
				if (f == 0 || (x & ~RS_FLAGS & ~0xFFFFFFFFull) != tag) {
					if (++spins > RS_SPIN_LIMIT) {
						atomicOr(err, RS_ERR_LOOKBACK);
						s_fail = 1;
						break;
					}
					__nanosleep(64);
					continue;
				}
				excl += x & 0xFFFFFFFFull;
				if (f == RS_PREFIX)
					break;
				t--;
			}
			st[(uint64_t) tile * 256 + d] = RS_PREFIX | tag | (excl + cnt);
		}
		uint32_t tot;
		const uint32_t hb = block_excl_scan<uint32_t>(hist[d], &tot, wsum);
		dstart[d] = block_excl_scan<uint32_t>(cnt, &tot, wsum);
		gbase[d] = hb + (uint32_t) excl;
	}
	__syncthreads();
	if (s_fail) {
		cp_async_wait_all();  // no copy may still target this CTA's shared memory
		return;
	}
#pragma unroll
	for (int i = 0; i < RS_ITEMS; i++) {
		const uint32_t local = (uint32_t) warp * (RS_ITEMS * 32) + i * 32 + lane;
		if (t0 + local < n) {
			const uint32_t d = rs_digit(k[i], shift);
			const uint32_t lp = dstart[d] + whist[warp * 256 + d] + loc[i];
			sk[lp] = k[i];
			si[lp] = (uint16_t) local;
		}
	}
	cp_async_wait_all();
	__syncthreads();
	for (uint32_t j = threadIdx.x; j < tile_n; j += RS_THREADS) {
		const K key = sk[j];
		const uint32_t d = rs_digit(key, shift);
		const uint64_t g = (uint64_t) gbase[d] + (j - dstart[d]);
		if (g < n) {
			keys_out[g] = key;
			vals_out[g] = vals_in ? sv[si[j]] : (V) (t0 + si[j]);
		}
	}
}

template <typename K, typename V>
constexpr size_t rs_onesweep_smem()
{
	return RS_TILE * (sizeof(K) + sizeof(V) + 2) + (RS_WARPS * 256 + 256 + 256 + 33) * 4;
}

inline uint64_t rs_num_tiles(uint64_t n) { return (n + RS_TILE - 1) / RS_TILE; }

// Scratch of radix_sort: key/value ping-pong buffers of n entries, the look-back
// status of every (tile, digit) and the small per-pass counters.  `status` must be
// zeroed once before the first sort that uses it; `epoch` then tags every pass so
// later sorts reuse it without clearing.
struct SortScratch {
	void *keys_alt = nullptr;  // n keys
	void *vals_alt = nullptr;  // n payloads
	void *vals_tmp = nullptr;  // n payloads (second buffer for an identity input payload)
	uint64_t *status = nullptr;  // rs_num_tiles(n) * 256
	uint32_t *hist = nullptr;    // RS_MAX_PASSES * 256, zeroed by radix_sort
	uint32_t *counters = nullptr;  // RS_MAX_PASSES tile counters, zeroed by radix_sort
	uint32_t *err = nullptr;
	uint32_t epoch = 1;
};

constexpr size_t rs_misc_words() { return RS_MAX_PASSES * 256 + RS_MAX_PASSES; }

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
// scratch ones; *vals_res stays null when passes == 0 and vals is null).  `hist` and
// `counters` must be adjacent (rs_misc_words()).  pre_hist (optional): the keys'
// digit counts, already made (pre_hist[p * 256 + v] = keys whose digit p is v), in
// place of the histogram pass.
template <typename K, typename V>
void radix_sort(K *keys, V *vals, uint64_t n, int passes, SortScratch &sc, K **keys_res, V **vals_res, cudaStream_t s,
                const uint32_t *pre_hist = nullptr)
{
	*keys_res = keys;
	*vals_res = vals;
	if (n == 0 || passes == 0)
		return;
	if (passes > RS_MAX_PASSES)
		fail(PST_ERR_INTERNAL, "radix sort: too many passes");
	const uint64_t tiles = rs_num_tiles(n);
	PST_CUDA(cudaFuncSetAttribute(k_rs_onesweep<K, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                              (int) rs_onesweep_smem<K, V>()));
	PST_CUDA(cudaMemsetAsync(sc.hist, 0, rs_misc_words() * 4, s));
	const unsigned hg = (unsigned) std::min<uint64_t>((n + RS_THREADS - 1) / RS_THREADS,
	                                                  (uint64_t) device_info().sms * 4);
	if (!pre_hist)
		k_rs_global_hist<K><<<hg, RS_THREADS, 4 * passes * 256 * 4, s>>>(keys, n, passes, sc.hist);
	const uint32_t *hist = pre_hist ? pre_hist : sc.hist;
	K *kin = keys, *kout = static_cast<K *>(sc.keys_alt);
	V *vin = vals;
	V *vout = static_cast<V *>(sc.vals_alt);
	for (int p = 0; p < passes; p++) {
		k_rs_onesweep<K, V><<<(unsigned) tiles, RS_THREADS, rs_onesweep_smem<K, V>(), s>>>(
		    kin, vin, kout, vout, n, 8 * p, hist + 256 * p, sc.status, sc.counters + p, sc.epoch++, sc.err);
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
