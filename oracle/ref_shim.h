/*
 * ref_shim.h — force-included (nvcc -include) when the reference's own CUDA
 * sources are compiled into oracle/_ref.  TEST INFRASTRUCTURE ONLY.
 *
 * It leaves the reference sources untouched and changes one thing: every
 * cudaMalloc in those translation units gets REF_SHIM_PAD bytes of zeroed
 * slack after the requested size.  The reference reads and writes one
 * element past some of its own arrays:
 *   - analysis/analysis_csr.cu:127 tests `groupId > n` instead of `>=`, so
 *     the tile with groupId == n writes dfr_analysis_info[n] and
 *     is_solved[n] (:181, :183), arrays allocated with n entries (:284-285);
 *   - solver/solve_csr_multirow.cu:47 reads iorder[base_idx + vect_idx]
 *     before the bounds check at :50 (up to 31 entries past the end of the
 *     n-entry iorder allocated at analysis_csr.cu:388).
 * With the slack those accesses stay inside the allocation they belong to.
 * The harness also records the allocations made during one analysis call, so
 * it can read back the level array the reference computes and leaks
 * (analysis_csr.cu:284, written by the level kernel at :181).
 */
#ifndef SPTRSV_REF_SHIM_H
#define SPTRSV_REF_SHIM_H

#include <cuda_runtime.h>
#include <stddef.h>

#define REF_SHIM_PAD 4096

#ifdef __cplusplus
extern "C" {
#endif
cudaError_t ref_shim_cudaMalloc(void** p, size_t bytes);
#ifdef __cplusplus
}
#endif

#define cudaMalloc(p, s) ref_shim_cudaMalloc((void**)(p), (size_t)(s))

#endif
