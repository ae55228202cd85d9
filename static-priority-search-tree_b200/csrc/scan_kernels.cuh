// Streaming kernels (interval parallel search, metacell formation): host entry points.
#pragma once

#include "common.cuh"

namespace pst {

// Writes up to `cap` matches of dim1 <= v <= dim2 to out and adds the number of
// matches to *counter_d (which the caller zeroes).
void ips_run(pst_dtype dt, pst_idtype it, pst_ret ret, const void *pts, uint64_t n, pst_value v, void *out,
             uint64_t cap, unsigned long long *counter_d, uint32_t blocks, cudaStream_t s);

// One record per metacell; M = metacell grid dims.
void metacells_run(pst_dtype dt, pst_idtype it, const void *vol, const uint32_t P[3], const uint32_t mc[3],
                   const uint32_t M[3], void *out, cudaStream_t s);
// Metacell layers [mz_begin, mz_end) only; `vol` points at vertex plane mz_begin * mc[2].
void metacells_run_layers(pst_dtype dt, pst_idtype it, const void *vol, const uint32_t P[3], const uint32_t mc[3],
                          const uint32_t M[3], uint32_t mz_begin, uint32_t mz_end, void *out, cudaStream_t s);

// Raw volume files streamed to the device (ingest.cu).
void read_volume(const char *path, pst_dtype dt, uint64_t num_vertices, void *vert_d, cudaStream_t s);
void metacells_from_file(const char *path, pst_dtype dt, pst_idtype it, const uint32_t P[3], const uint32_t mc[3],
                         const uint32_t M[3], void *out_d, uint64_t slab_bytes, cudaStream_t s);

}  // namespace pst
