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

}  // namespace pst
