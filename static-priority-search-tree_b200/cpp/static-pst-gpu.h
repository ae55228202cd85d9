// C++ facade with the reference's template surface, over the C ABI of
// libpst_b200.so (include/pst_c.h).  Header-only; link with -lpst_b200 -lcudart.
//
// Re-creates, with the same names, template parameters, argument order and
// conventions (callee-allocated device results freed by the caller with cudaFree,
// blocking searches, std::runtime_error on failure, "Tree is empty; nothing to
// search" for empty trees):
//   StaticPSTGPU     pst/static-pst-gpu.h:69-165
//   StaticPSTGPUArr  pst/static-pst-gpu-arr.h:45-103
//   intervalParallelSearch  interval-parallel-search/interval-parallel-search.h:23-66
//   calcNumMetacells / formMetacellTags / formVoxelTags
//                    helpers/isosurface-data-processing.h:21-203
// The PointStruct template and the StaticPrioritySearchTree base are provided by
// pst-b200-compat.h when the reference's own headers are not already included.
#ifndef PST_B200_STATIC_PST_GPU_H
#define PST_B200_STATIC_PST_GPU_H

#include <cuda_runtime.h>

#include <cstring>
#include <iostream>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "pst-b200-compat.h"
#include "pst_c.h"

namespace pst_b200_detail {

template <typename T>
constexpr pst_dtype dtype_of()
{
	static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value || std::is_same<T, int>::value,
	              "supported value types: float, double, int");
	return std::is_same<T, float>::value ? PST_F32 : std::is_same<T, double>::value ? PST_F64 : PST_I32;
}

template <typename IDType, size_t num_IDs>
constexpr pst_idtype idtype_of()
{
	static_assert(num_IDs == 0 || (num_IDs == 1 && sizeof(IDType) == 4 && std::is_integral<IDType>::value),
	              "supported ids: none, or one 32-bit integer id");
	return num_IDs == 0 ? PST_ID_NONE : PST_ID_U32;
}

template <typename T>
pst_value to_value(T v)
{
	pst_value x;
	std::memset(&x, 0, sizeof(x));
	if constexpr (std::is_same<T, float>::value)
		x.f32 = v;
	else if constexpr (std::is_same<T, double>::value)
		x.f64 = v;
	else
		x.i32 = v;
	return x;
}

inline void check(pst_status st, const std::string &what)
{
	if (st != PST_OK)
		throw std::runtime_error(what + ": " + pst_last_error());
}

}  // namespace pst_b200_detail

template <typename T, template <typename, typename, size_t> class PointStructTemplate, typename IDType = void,
          size_t num_IDs = 0>
class StaticPSTGPU : public StaticPrioritySearchTree<T, PointStructTemplate, IDType, num_IDs>
{
  public:
	using Point = PointStructTemplate<T, IDType, num_IDs>;

	// warp_multiplier and dev_props are launch hints of the reference; this
	// implementation sizes its grids itself.  dev_ind selects the device.
	StaticPSTGPU(Point *const pt_arr_d, size_t num_elems, const int warp_multiplier = 1, int dev_ind = 0,
	             int num_devs = 1, cudaDeviceProp dev_props = {})
	    : num_elems(num_elems), dev_ind(dev_ind), num_devs(num_devs), dev_props(dev_props)
	{
		(void) warp_multiplier;
		static_assert(sizeof(Point) == (num_IDs ? (sizeof(T) == 8 ? 24 : 12) : 2 * sizeof(T)),
		              "PointStruct layout must match the reference's");
		pst_b200_detail::check(cudaSetDevice(dev_ind) == cudaSuccess ? PST_OK : PST_ERR_CUDA,
		                       "Error in selecting device " + std::to_string(dev_ind + 1) + " (1-indexed) of " +
		                           std::to_string(num_devs));
		pst_b200_detail::check(pst_create(&tree, pst_b200_detail::dtype_of<T>(),
		                                  pst_b200_detail::idtype_of<IDType, num_IDs>(), pt_arr_d, num_elems, nullptr),
		                       "Error in constructing priority search tree on device " + std::to_string(dev_ind + 1) +
		                           " (1-indexed) of " + std::to_string(num_devs));
	}

	virtual ~StaticPSTGPU() { pst_destroy(tree); }

	StaticPSTGPU(const StaticPSTGPU &) = delete;
	StaticPSTGPU &operator=(const StaticPSTGPU &) = delete;

	virtual void print(std::ostream &os) const
	{
		if (num_elems == 0) {
			os << "Tree is empty\n";
			return;
		}
		uint64_t slots = 0;
		pst_b200_detail::check(pst_info(tree, nullptr, nullptr, &slots, nullptr, nullptr, nullptr), "pst_info");
		std::vector<T> d1(slots), d2(slots), md(slots);
		std::vector<uint32_t> ids(slots);
		std::vector<uint8_t> bc(slots);
		pst_b200_detail::check(pst_export(tree, d1.data(), d2.data(), md.data(), ids.data(), bc.data()), "pst_export");
		print_recur(os, d1, d2, md, ids, bc, 0, "", "");
	}

	int getDevInd() const { return dev_ind; }
	cudaDeviceProp getDevProps() const { return dev_props; }
	int getNumDevs() const { return num_devs; }

	template <typename RetType = Point>
	    requires std::disjunction<std::is_same<RetType, IDType>, std::is_same<RetType, Point>>::value
	void threeSidedSearch(size_t &num_res_elems, RetType *&res_arr_d, T min_dim1_val, T max_dim1_val, T min_dim2_val,
	                      const int warp_multiplier = 1)
	{
		(void) warp_multiplier;
		search<RetType>(PST_Q_THREE, num_res_elems, res_arr_d, min_dim1_val, max_dim1_val, min_dim2_val);
	}

	template <typename RetType = Point>
	    requires std::disjunction<std::is_same<RetType, IDType>, std::is_same<RetType, Point>>::value
	void twoSidedLeftSearch(size_t &num_res_elems, RetType *&res_arr_d, T max_dim1_val, T min_dim2_val,
	                        const int warp_multiplier = 1)
	{
		(void) warp_multiplier;
		search<RetType>(PST_Q_LEFT, num_res_elems, res_arr_d, T(0), max_dim1_val, min_dim2_val);
	}

	template <typename RetType = Point>
	    requires std::disjunction<std::is_same<RetType, IDType>, std::is_same<RetType, Point>>::value
	void twoSidedRightSearch(size_t &num_res_elems, RetType *&res_arr_d, T min_dim1_val, T min_dim2_val,
	                         const int warp_multiplier = 1)
	{
		(void) warp_multiplier;
		search<RetType>(PST_Q_RIGHT, num_res_elems, res_arr_d, min_dim1_val, T(0), min_dim2_val);
	}

	static size_t calcGlobalMemNeeded(const size_t num_elems)
	{
		uint64_t b = 0;
		pst_b200_detail::check(pst_mem_needed(pst_b200_detail::dtype_of<T>(),
		                                      pst_b200_detail::idtype_of<IDType, num_IDs>(), num_elems, &b),
		                       "pst_mem_needed");
		return (size_t) b;
	}

	pst_tree *handle() const { return tree; }

  protected:
	template <typename RetType>
	void search(pst_qkind kind, size_t &num_res_elems, RetType *&res_arr_d, T a, T b, T c)
	{
		if (num_elems == 0) {
			std::cout << "Tree is empty; nothing to search\n";
			num_res_elems = 0;
			res_arr_d = nullptr;
			return;
		}
		pst_query q;
		std::memset(&q, 0, sizeof(q));
		q.kind = kind;
		q.min1 = pst_b200_detail::to_value(a);
		q.max1 = pst_b200_detail::to_value(b);
		q.min2 = pst_b200_detail::to_value(c);
		void *out = nullptr;
		uint64_t cnt = 0;
		const pst_ret ret = std::is_same<RetType, Point>::value ? PST_RET_POINTS : PST_RET_IDS;
		pst_b200_detail::check(pst_search(tree, &q, ret, &out, &cnt, nullptr),
		                       "Error in searching on device " + std::to_string(dev_ind + 1) + " (1-indexed) of " +
		                           std::to_string(num_devs));
		num_res_elems = (size_t) cnt;
		res_arr_d = static_cast<RetType *>(out);
	}

	void print_recur(std::ostream &os, const std::vector<T> &d1, const std::vector<T> &d2, const std::vector<T> &md,
	                 const std::vector<uint32_t> &ids, const std::vector<uint8_t> &bc, size_t i, std::string prefix,
	                 std::string child_prefix) const
	{
		os << prefix << '(' << d1[i] << ", " << d2[i] << "; " << md[i];
		if constexpr (num_IDs == 1)
			os << "; " << ids[i];
		os << ')';
		const bool l = bc[i] & 0x2, r = bc[i] & 0x1;
		if (l && r) {
			print_recur(os, d1, d2, md, ids, bc, 2 * i + 2, '\n' + child_prefix + "├─(R)─ ", child_prefix + "│      ");
			print_recur(os, d1, d2, md, ids, bc, 2 * i + 1, '\n' + child_prefix + "└─(L)─ ", child_prefix + "       ");
		} else if (r) {
			print_recur(os, d1, d2, md, ids, bc, 2 * i + 2, '\n' + child_prefix + "└─(R)─ ", child_prefix + "       ");
		} else if (l) {
			print_recur(os, d1, d2, md, ids, bc, 2 * i + 1, '\n' + child_prefix + "└─(L)─ ", child_prefix + "       ");
		}
	}

	pst_tree *tree = nullptr;
	size_t num_elems;
	int dev_ind;
	int num_devs;
	cudaDeviceProp dev_props;
};

// The reference's array-of-shallow-trees variant (pst/static-pst-gpu-arr.h:45-103).
// Its searches run on one complete tree here, so threeSidedSearch and
// twoSidedRightSearch (empty bodies in the reference, pst/static-pst-gpu-arr.tu:571-578,
// :652-658) return the full, correct result as well.
template <typename T, template <typename, typename, size_t> class PointStructTemplate, typename IDType = void,
          size_t num_IDs = 0>
class StaticPSTGPUArr : public StaticPSTGPU<T, PointStructTemplate, IDType, num_IDs>
{
  public:
	using Base = StaticPSTGPU<T, PointStructTemplate, IDType, num_IDs>;
	StaticPSTGPUArr(typename Base::Point *const pt_arr_d, const size_t num_elems, const unsigned threads_per_block,
	                const int dev_ind = 0, const int num_devs = 1, const cudaDeviceProp &dev_props = {})
	    : Base(pt_arr_d, num_elems, 1, dev_ind, num_devs, dev_props), threads_per_block(threads_per_block)
	{
	}

	template <typename RetType = typename Base::Point>
	void threeSidedSearch(size_t &num_res_elems, RetType *&res_arr_d, const T min_dim1_val, const T max_dim1_val,
	                      const T min_dim2_val)
	{
		Base::template threeSidedSearch<RetType>(num_res_elems, res_arr_d, min_dim1_val, max_dim1_val, min_dim2_val);
	}
	template <typename RetType = typename Base::Point>
	void twoSidedLeftSearch(size_t &num_res_elems, RetType *&res_arr_d, const T max_dim1_val, const T min_dim2_val)
	{
		Base::template twoSidedLeftSearch<RetType>(num_res_elems, res_arr_d, max_dim1_val, min_dim2_val);
	}
	template <typename RetType = typename Base::Point>
	void twoSidedRightSearch(size_t &num_res_elems, RetType *&res_arr_d, const T min_dim1_val, const T min_dim2_val)
	{
		Base::template twoSidedRightSearch<RetType>(num_res_elems, res_arr_d, min_dim1_val, min_dim2_val);
	}

	static size_t calcGlobalMemNeeded(const size_t num_elems, const unsigned threads_per_block)
	{
		(void) threads_per_block;
		return Base::calcGlobalMemNeeded(num_elems);
	}

  private:
	unsigned threads_per_block;
};

// interval-parallel-search/interval-parallel-search.h:23-66
template <typename T, template <typename, typename, size_t> class PointStructTemplate, typename IDType, size_t num_IDs,
          typename RetType>
    requires std::disjunction<std::is_same<RetType, IDType>,
                              std::is_same<RetType, PointStructTemplate<T, IDType, num_IDs>>>::value
void intervalParallelSearch(PointStructTemplate<T, IDType, num_IDs> *pt_arr_d, const size_t num_elems,
                            RetType *&res_arr_d, size_t &num_res_elems, T search_val, const int dev_ind,
                            const int num_devs, const int warp_size, const unsigned num_thread_blocks,
                            const unsigned threads_per_block)
{
	(void) warp_size;
	void *out = nullptr;
	uint64_t cnt = 0;
	const pst_ret ret =
	    std::is_same<RetType, PointStructTemplate<T, IDType, num_IDs>>::value ? PST_RET_POINTS : PST_RET_IDS;
	pst_b200_detail::check(pst_ips_search(pst_b200_detail::dtype_of<T>(), pst_b200_detail::idtype_of<IDType, num_IDs>(),
	                                      pt_arr_d, num_elems, pst_b200_detail::to_value(search_val), ret, &out, &cnt,
	                                      num_thread_blocks, threads_per_block, nullptr),
	                       "Error in interval parallel search on device " + std::to_string(dev_ind + 1) +
	                           " (1-indexed) of " + std::to_string(num_devs));
	res_arr_d = static_cast<RetType *>(out);
	num_res_elems = (size_t) cnt;
}

// helpers/isosurface-data-processing.h:21-36
template <typename GridDimType>
    requires std::is_integral<GridDimType>::value
void calcNumMetacells(GridDimType pt_grid_dims[3], GridDimType metacell_dims[3], GridDimType metacell_grid_dims[3],
                      size_t &num_metacells)
{
	uint32_t p[3], m[3], g[3];
	for (int i = 0; i < 3; i++) {
		p[i] = (uint32_t) pt_grid_dims[i];
		m[i] = (uint32_t) metacell_dims[i];
	}
	uint64_t n = 0;
	pst_b200_detail::check(pst_num_metacells(p, m, g, &n), "calcNumMetacells");
	for (int i = 0; i < 3; i++)
		metacell_grid_dims[i] = (GridDimType) g[i];
	num_metacells = (size_t) n;
}

// helpers/isosurface-data-processing.h:66-137 (the result is cudaMalloc'd; the caller frees it)
template <class PointStruct, typename T, typename GridDimType>
PointStruct *formMetacellTags(T *const vertex_arr_d, GridDimType pt_grid_dims[3], GridDimType metacell_dims[3],
                              GridDimType metacell_grid_dims[3], const size_t num_metacells, const int dev_ind,
                              const int num_devs, const int warp_size)
{
	(void) metacell_grid_dims;
	(void) warp_size;
	PointStruct *out = nullptr;
	if (cudaMalloc(&out, num_metacells * sizeof(PointStruct)) != cudaSuccess)
		throw std::runtime_error("Error in allocating metacell tag storage array on device " +
		                         std::to_string(dev_ind + 1) + " (1-indexed) of " + std::to_string(num_devs));
	uint32_t p[3], m[3];
	for (int i = 0; i < 3; i++) {
		p[i] = (uint32_t) pt_grid_dims[i];
		m[i] = (uint32_t) metacell_dims[i];
	}
	constexpr bool has_id = sizeof(PointStruct) > 2 * sizeof(T);
	const pst_status st = pst_form_metacells(pst_b200_detail::dtype_of<T>(), has_id ? PST_ID_U32 : PST_ID_NONE,
	                                         vertex_arr_d, p, m, out, nullptr);
	if (st != PST_OK) {
		cudaFree(out);
		pst_b200_detail::check(st, "Error in forming metacell tags");
	}
	return out;
}

// helpers/isosurface-data-processing.h:139-203: one tag per voxel (metacells of 1^3 voxels)
template <class PointStruct, typename T, typename GridDimType>
PointStruct *formVoxelTags(T *const vertex_arr_d, GridDimType pt_grid_dims[3], GridDimType metacell_dims[3],
                           size_t &num_voxels, const int dev_ind, const int num_devs)
{
	(void) metacell_dims;
	GridDimType ones[3] = {1, 1, 1}, grid[3];
	calcNumMetacells(pt_grid_dims, ones, grid, num_voxels);
	return formMetacellTags<PointStruct>(vertex_arr_d, pt_grid_dims, ones, grid, num_voxels, dev_ind, num_devs, 32);
}

#endif
