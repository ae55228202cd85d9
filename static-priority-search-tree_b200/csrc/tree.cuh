// Tree storage and the entry points of construction and search (host side).
#pragma once

#include <mutex>

#include "common.cuh"

namespace pst {

struct Batch;

// Owns the device arrays of one tree (see TreeDev for the layout).
struct TreeStorage {
	pst_dtype dtype = PST_F32;
	pst_idtype idtype = PST_ID_NONE;
	uint64_t n = 0;
	uint32_t levels = 0;
	void *mem = nullptr;  // single cudaMalloc holding every field
	size_t bytes = 0;
	void *dim1 = nullptr;
	void *dim2 = nullptr;
	void *med = nullptr;
	uint32_t *id = nullptr;
	uint32_t *occ = nullptr;
	uint32_t *last_par = nullptr;  // separate allocation, see TreeDev::last_par
	void *sub_min = nullptr;       // separate allocation, see TreeDev::sub_min
	int device = 0;
	std::mutex mu;        // serialises the single-query engine
	Batch *single = nullptr;

	template <typename T>
	TreeDev<T> view() const
	{
		return TreeDev<T>{static_cast<const T *>(dim1), static_cast<const T *>(dim2), static_cast<const T *>(med),
		                  id, occ, n, levels, last_par, static_cast<const T *>(sub_min)};
	}
};

size_t value_size(pst_dtype dt);
size_t point_size(pst_dtype dt, pst_idtype it);
// Device bytes of the tree arrays alone.
uint64_t tree_bytes(pst_dtype dt, pst_idtype it, uint64_t n);
// Tree arrays plus the peak construction working set.
uint64_t build_bytes_needed(pst_dtype dt, pst_idtype it, uint64_t n);
// Points the field pointers of t (dtype, idtype, n set) into one allocation of
// tree_bytes(...) bytes laid out as the builder lays it out.
void attach_tree_memory(TreeStorage &t, void *mem);
// Derives the auxiliary search indexes (TreeDev::last_par, TreeDev::sub_min) from
// the occupancy and the dim2 values.
void finish_tree_aux(TreeStorage &t, cudaStream_t s);
// Tree image: a 64-byte header followed by the device allocation byte for byte.
uint64_t serialized_size(const TreeStorage &t);
void save_tree(const TreeStorage &t, void *host, uint64_t capacity, cudaStream_t s);
void load_tree(TreeStorage &t, const void *host, uint64_t size, cudaStream_t s);
void save_tree_file(const TreeStorage &t, const char *path);
void load_tree_file(TreeStorage &t, const char *path, cudaStream_t s);
// Marching cubes over the cells of the given metacells (mc.cu).  Returns the
// triangle count; writes the triangles only when emit and they fit `capacity`.
void mc_tables(uint8_t *ntri, uint8_t *edges);
uint64_t mc_run(const float *vol, const uint32_t P[3], const uint32_t mc[3], const uint32_t *ids, uint64_t n, float iso,
                float *tri, uint64_t capacity, bool emit, cudaStream_t s);

void build_tree(TreeStorage &t, const void *pts_d, uint64_t n, cudaStream_t s);
void free_tree(TreeStorage &t);
// Host copy in the reference's field layout (slot = heap index - 1).
void export_tree(const TreeStorage &t, void *dim1, void *dim2, void *med, uint32_t *ids, uint8_t *bitcodes);

}  // namespace pst

// Opaque handle of the C ABI.
struct pst_tree {
	pst::TreeStorage t;
};
