// Shared definitions of the B200 static priority search tree library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "pst_c.h"

namespace pst {

// ---------------------------------------------------------------------------
// Errors.  Library code throws pst::Error internally; the C ABI layer turns it
// into a pst_status plus a thread-local message.

struct Error {
	pst_status status;
	std::string msg;
};

[[noreturn]] void fail(pst_status st, const std::string &msg);
void check_cuda(cudaError_t e, const char *what);

#define PST_CUDA(call) ::pst::check_cuda((call), #call)

// ---------------------------------------------------------------------------
// Point records: the reference's PointStruct layouts (helpers/point-struct.h).

template <typename T, bool HAS_ID>
struct Point;
template <typename T>
struct Point<T, true> {
	T dim1;
	T dim2;
	uint32_t id;
};
template <typename T>
struct Point<T, false> {
	T dim1;
	T dim2;
};

// ---------------------------------------------------------------------------
// Order-preserving unsigned keys.  Comparing keys as unsigned integers gives the
// order of the values under the C++ `<` of the reference's comparators
// (helpers/point-struct.h:62-81); -0.0 is mapped onto +0.0 because `!=` treats
// them as equal there, so ties between them fall to the id/index tiebreak.
// NaN inputs are outside the contract (the reference's comparators are not a
// strict weak order on them).

template <typename T>
struct KeyOf;

template <>
struct KeyOf<float> {
	using K = uint32_t;
	__host__ __device__ static K key(float v)
	{
		uint32_t u;
		memcpy(&u, &v, 4);
		if (v == 0.0f)
			u = 0;
		return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
	}
	// The value of a key (inverse of key() for every value but -0.0, whose key is
	// +0.0's).
	__host__ __device__ static float value(K k)
	{
		const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
		float v;
		memcpy(&v, &u, 4);
		return v;
	}
};

template <>
struct KeyOf<double> {
	using K = uint64_t;
	__host__ __device__ static K key(double v)
	{
		uint64_t u;
		memcpy(&u, &v, 8);
		if (v == 0.0)
			u = 0;
		return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
	}
	__host__ __device__ static double value(K k)
	{
		const uint64_t u = (k & 0x8000000000000000ull) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
		double v;
		memcpy(&v, &u, 8);
		return v;
	}
};

template <>
struct KeyOf<int32_t> {
	using K = uint32_t;
	__host__ __device__ static K key(int32_t v) { return static_cast<uint32_t>(v) ^ 0x80000000u; }
	__host__ __device__ static int32_t value(K k) { return static_cast<int32_t>(k ^ 0x80000000u); }
};

// ---------------------------------------------------------------------------
// Device tree.  Heap positions are 1-based (root = 1, children 2h and 2h+1), so
// level d occupies [2^d, 2^(d+1)) and every 32-slot chunk at levels >= 5 starts
// on a 128-byte boundary of a 4-byte field.  Arrays hold 2^levels entries
// (position 0 unused); med holds 2^(levels-1) (internal levels only).
// All levels but the last are full; occ has one bit per position.

template <typename T>
struct TreeDev {
	const T *dim1;
	const T *dim2;
	const T *med;
	const uint32_t *id;   // null for id-less trees
	const uint32_t *occ;  // occupancy bitmap, 2^levels bits
	uint64_t n;
	uint32_t levels;      // D = floor(log2 n) + 1
	// One bit per 64-slot block of level D-2: does any of its children exist?
	// (null when D-2 < 6).  A sparse last level lets the last expansion skip the
	// records whose blocks have no children before reading their occupancy.
	const uint32_t *last_par;
	// Per 64-slot block of levels 6..D-2 (index = its first position / 64): the
	// smallest dim2 among all the block's descendants (NaN if any is NaN; null when
	// D < 8).  A query whose min2 is at most this value reports every descendant of
	// the block's reported slots, so their dim2 need no test.
	const T *sub_min;
};

// Number of levels of a tree of n points: floor(log2 n) + 1 (0 for n == 0).
inline uint32_t tree_levels(uint64_t n)
{
	uint32_t d = 0;
	while ((n >> d) != 0)
		d++;
	return d;
}

// Point count of the node at level d, index j within the level.  Construction
// gives a node of c points a left child of floor(c/2) and a right child of
// c - 1 - floor(c/2) points (pst/static-pst-cpu-iter.tpp:512-541), so counts
// depend on n and the node's path only.
__host__ __device__ inline uint64_t node_count(uint64_t n, uint32_t d, uint64_t j)
{
	uint64_t c = n;
	for (int b = (int) d - 1; b >= 0 && c != 0; b--)
		c = ((j >> b) & 1) ? c - 1 - c / 2 : c / 2;
	return c;
}

// ---------------------------------------------------------------------------
// Warp helpers.

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

// Spreads the 16 low bits of x so that bit j lands on bits 2j and 2j+1: the
// children of the 16 parents of a half chunk fill one whole chunk.
__host__ __device__ __forceinline__ uint32_t spread16(uint32_t x)
{
	x &= 0xFFFFu;
	x = (x | (x << 8)) & 0x00FF00FFu;
	x = (x | (x << 4)) & 0x0F0F0F0Fu;
	x = (x | (x << 2)) & 0x33333333u;
	x = (x | (x << 1)) & 0x55555555u;
	return x | (x << 1);
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v)
{
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		T t = __shfl_up_sync(0xFFFFFFFFu, v, o);
		if ((int) lane_id() >= o)
			v += t;
	}
	return v;
}

// Segmented inclusive sum over lanes whose `key` equals the previous lane's key
// (runs of equal keys).  Returns the run-inclusive sum; *last is true on the last
// lane of each run.
__device__ __forceinline__ uint64_t warp_run_sum(uint32_t key, uint64_t v, bool *last)
{
	const uint32_t lane = lane_id();
	uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, key, 1);
	uint32_t head = (lane == 0 || prev != key) ? 1u : 0u;
	uint32_t heads = __ballot_sync(0xFFFFFFFFu, head);
	// start lane of my run = highest head lane <= lane
	uint32_t mask_le = heads & (0xFFFFFFFFu >> (31 - lane));
	uint32_t start = 31 - __clz(mask_le);
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint64_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
		if (lane >= start + o)
			v += t;
	}
	uint32_t next = __shfl_down_sync(0xFFFFFFFFu, key, 1);
	*last = (lane == 31) || (next != key);
	return v;
}

// Asynchronous global -> shared copies (cp.async): 16 or 4 bytes per thread, in
// commit groups; wait_group<N> waits until at most N of this thread's groups are
// still in flight.
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
	             "l"(src)
	             : "memory");
}

__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
	asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
	             "l"(src)
	             : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group()
{
	asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Per-stream device facts used for grid sizing.
struct DeviceInfo {
	int device;
	int sms;
	size_t smem_optin;
};
const DeviceInfo &device_info();

}  // namespace pst
