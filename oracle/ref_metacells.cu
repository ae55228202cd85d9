// TEST INFRASTRUCTURE ONLY: the reference's own metacell formation
// (formMetacellTags / formMetacellTagsGlobal / getVoxelMinMax,
// helpers/isosurface-data-processing.h:23-137, helpers/isosurface-data-processing.tu:9-127,
// :181-212), compiled unmodified from the reference's sources into
// oracle/_ref/libmcref.so, so that the GPU tests can pin the oracle's metacell
// restatement to the reference itself.  No product code path links or calls it.
//
// The reference does not compile as it stands with CUDA 12.9: its kernel passes the
// overloaded names `min` and `max` to cooperative_groups::reduce, which cannot pick
// an overload from a set.  This translation unit includes every header those
// sources need first, then makes `min` and `max` name function objects (a
// preprocessor shim: the reference's files are not changed), then includes the
// reference's header, which pulls in its .tu.  The function objects keep the
// reference's meaning: on the device the CUDA math min/max of the value type (fminf,
// fmaxf, fmin, fmax for floating point, integer min/max otherwise), on the host
// std::min / std::max.
//
// Inputs the reference handles: point dims P and metacell dims mc (one block of
// mc threads per metacell) such that
//   - (P - 1) mod mc != 0 on every axis: its grid-stride loops step by
//     ceil((P - 1) / mc) * mc, so with a zero remainder they run a second pass in
//     which every block leader writes a metacell id past the grid;
//   - the first thread of every warp of a block lies on a valid voxel in the last
//     metacell of each axis (which holds (P - 1) mod mc voxels there): a warp whose
//     first lane has no voxel hands an uninitialised min/max to the inter-warp
//     reduction.
// The entry point below rejects other sizes (returns -1) without launching anything.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <nvfunctional>
#include <string>
#include <type_traits>

#include "calc-alloc-report-ind-offset.h"
#include "class-member-checkers.h"
#include "dev-symbols.h"  // after calc-alloc-report-ind-offset.h, in the reference's own order
#include "exit-status-codes.h"
#include "gpu-err-chk.h"
#include "linearise-id.h"
#include "point-struct.h"
#include "type-concepts.h"

struct PstRefMinFn {
	template <typename A, typename B>
	__host__ __device__ constexpr auto operator()(A a, B b) const
	{
#ifdef __CUDA_ARCH__
		if constexpr (std::is_same_v<A, float> && std::is_same_v<B, float>)
			return fminf(a, b);
		else if constexpr (std::is_same_v<A, double> && std::is_same_v<B, double>)
			return fmin(a, b);
		else
			return (b < a) ? b : a;
#else
		return (b < a) ? b : a;
#endif
	}
};

struct PstRefMaxFn {
	template <typename A, typename B>
	__host__ __device__ constexpr auto operator()(A a, B b) const
	{
#ifdef __CUDA_ARCH__
		if constexpr (std::is_same_v<A, float> && std::is_same_v<B, float>)
			return fmaxf(a, b);
		else if constexpr (std::is_same_v<A, double> && std::is_same_v<B, double>)
			return fmax(a, b);
		else
			return (a < b) ? b : a;
#else
		return (a < b) ? b : a;
#endif
	}
};

// Object names the shim maps `min` / `max` to: device objects in the device
// compilation pass (the kernel's calls), host objects in the host pass, there also
// in std (the host code's std::min / std::max).
__device__ constexpr PstRefMinFn pst_ref_min_dev{};
__device__ constexpr PstRefMaxFn pst_ref_max_dev{};
inline constexpr PstRefMinFn pst_ref_min_obj{};
inline constexpr PstRefMaxFn pst_ref_max_obj{};
namespace std {
using ::pst_ref_max_dev;
using ::pst_ref_max_obj;
using ::pst_ref_min_dev;
using ::pst_ref_min_obj;
}  // namespace std

#ifdef __CUDA_ARCH__
#define min pst_ref_min_dev
#define max pst_ref_max_dev
#else
#define min pst_ref_min_obj
#define max pst_ref_max_obj
#endif
#include "isosurface-data-processing.h"
#undef min
#undef max

namespace {

template <typename T>
int64_t run(const void *vol_d, const uint32_t P[3], const uint32_t mc[3], void *out_d)
{
	for (int i = 0; i < 3; i++)
		if (P[i] < 2 || mc[i] == 0 || mc[i] > 64 || (P[i] - 1) % mc[i] == 0)
			return -1;  // a size the reference's kernel mishandles (see above): not launched
	const uint64_t threads = uint64_t(mc[0]) * mc[1] * mc[2];
	if (threads > 1024)
		return -1;
	for (uint64_t t = 32; t < threads; t += 32) {
		// first thread of a warp: (x, y, z) inside the block
		const uint64_t tx = t % mc[0], ty = (t / mc[0]) % mc[1], tz = t / (uint64_t(mc[0]) * mc[1]);
		if (tx >= (P[0] - 1) % mc[0] || ty >= (P[1] - 1) % mc[1] || tz >= (P[2] - 1) % mc[2])
			return -1;
	}
	int pt[3] = {int(P[0]), int(P[1]), int(P[2])};
	int md[3] = {int(mc[0]), int(mc[1]), int(mc[2])};
	int grid[3];
	size_t n = 0;
	calcNumMetacells(pt, md, grid, n);
	using PS = PointStruct<T, uint32_t, 1>;
	PS *res = formMetacellTags<PS>(static_cast<T *>(const_cast<void *>(vol_d)), pt, md, grid, n, 0, 1, 32);
	if (cudaDeviceSynchronize() != cudaSuccess)
		return -2;
	if (cudaMemcpy(out_d, res, n * sizeof(PS), cudaMemcpyDeviceToDevice) != cudaSuccess)
		return -2;
	cudaFree(res);
	return int64_t(n);
}

}  // namespace

// Metacell records (PointStruct<T, uint32_t, 1>: min, max, id) of a device volume
// (x fastest) into out_d (device, one record per metacell, indexed by id).  Returns
// the number of metacells, -1 for a size the reference mishandles (nothing run),
// -2 for a CUDA error.
extern "C" int64_t ref_metacells(int dtype, const void *vol_d, const uint32_t P[3], const uint32_t mc[3], void *out_d)
{
	switch (dtype) {
	case 0: return run<float>(vol_d, P, mc, out_d);
	case 1: return run<double>(vol_d, P, mc, out_d);
	case 2: return run<int32_t>(vol_d, P, mc, out_d);
	}
	return -1;
}
