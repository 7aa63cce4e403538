/*
 * cusparse_cmp.cu — cuSPARSE SpSV comparator for the benchmark.
 *
 * TEST AND BENCHMARK INFRASTRUCTURE ONLY.  The reference wraps cuSPARSE's
 * csrsv2 solve (solver/solve_csr_cusparse.cu:4-29), an API that no longer
 * exists in CUDA 12.9; its successor is cusparseSpSV.  This times the
 * solve phase only, as the reference wrapper does (:10-23), FP64, on the
 * same CSR (lower triangular, non-unit diagonal).
 */
#include <cuda_runtime.h>
#include <cusparse.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#define CK(x)                                                                   \
    do {                                                                        \
        cudaError_t e_ = (x);                                                   \
        if (e_ != cudaSuccess) {                                                \
            fprintf(stderr, "cuda %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return -4;                                                          \
        }                                                                       \
    } while (0)
#define CS(x)                                                                   \
    do {                                                                        \
        cusparseStatus_t s_ = (x);                                              \
        if (s_ != CUSPARSE_STATUS_SUCCESS) {                                    \
            fprintf(stderr, "cusparse %d at %s:%d\n", (int)s_, __FILE__, __LINE__); \
            return -5;                                                          \
        }                                                                       \
    } while (0)

extern "C" int cmp_cusparse_spsv(int n, const int* rowptr, const int* col, const double* val, const double* b,
                                 double* x, int reps, float* solve_ms, float* analysis_ms)
{
    const int nnz = rowptr[n];
    int *d_rp = nullptr, *d_ci = nullptr;
    double *d_va = nullptr, *d_b = nullptr, *d_x = nullptr;
    void* buf = nullptr;
    CK(cudaMalloc((void**)&d_rp, sizeof(int) * (n + 1)));
    CK(cudaMalloc((void**)&d_ci, sizeof(int) * nnz));
    CK(cudaMalloc((void**)&d_va, sizeof(double) * nnz));
    CK(cudaMalloc((void**)&d_b, sizeof(double) * n));
    CK(cudaMalloc((void**)&d_x, sizeof(double) * n));
    CK(cudaMemcpy(d_rp, rowptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_ci, col, sizeof(int) * nnz, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_va, val, sizeof(double) * nnz, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_b, b, sizeof(double) * n, cudaMemcpyHostToDevice));
    cusparseHandle_t h;
    CS(cusparseCreate(&h));
    cusparseSpMatDescr_t A;
    cusparseDnVecDescr_t vb, vx;
    cusparseSpSVDescr_t sv;
    CS(cusparseCreateCsr(&A, n, n, nnz, d_rp, d_ci, d_va, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                         CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F));
    cusparseFillMode_t fill = CUSPARSE_FILL_MODE_LOWER;
    cusparseDiagType_t diag = CUSPARSE_DIAG_TYPE_NON_UNIT;
    CS(cusparseSpMatSetAttribute(A, CUSPARSE_SPMAT_FILL_MODE, &fill, sizeof(fill)));
    CS(cusparseSpMatSetAttribute(A, CUSPARSE_SPMAT_DIAG_TYPE, &diag, sizeof(diag)));
    CS(cusparseCreateDnVec(&vb, n, d_b, CUDA_R_64F));
    CS(cusparseCreateDnVec(&vx, n, d_x, CUDA_R_64F));
    CS(cusparseSpSV_createDescr(&sv));
    const double alpha = 1.0;
    size_t bsz = 0;
    CS(cusparseSpSV_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A, vb, vx, CUDA_R_64F,
                               CUSPARSE_SPSV_ALG_DEFAULT, sv, &bsz));
    CK(cudaMalloc(&buf, bsz > 0 ? bsz : 1));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    CS(cusparseSpSV_analysis(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A, vb, vx, CUDA_R_64F,
                             CUSPARSE_SPSV_ALG_DEFAULT, sv, buf));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float am = 0;
    cudaEventElapsedTime(&am, e0, e1);
    std::vector<float> ts;
    for (int r = 0; r < (reps < 1 ? 1 : reps) + 1; r++) {
        cudaEventRecord(e0);
        CS(cusparseSpSV_solve(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A, vb, vx, CUDA_R_64F,
                              CUSPARSE_SPSV_ALG_DEFAULT, sv));
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0) ts.push_back(ms);  // first solve is a warm-up
    }
    std::sort(ts.begin(), ts.end());
    CK(cudaMemcpy(x, d_x, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (solve_ms) *solve_ms = ts[ts.size() / 2];
    if (analysis_ms) *analysis_ms = am;
    cusparseSpSV_destroyDescr(sv);
    cusparseDestroyDnVec(vb);
    cusparseDestroyDnVec(vx);
    cusparseDestroySpMat(A);
    cusparseDestroy(h);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    cudaFree(d_rp);
    cudaFree(d_ci);
    cudaFree(d_va);
    cudaFree(d_b);
    cudaFree(d_x);
    return 0;
}
