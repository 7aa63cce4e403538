// solve.cu — host side of the solves: the reference entry points
// (header/solver.h:5-7) over the caller's CSR, and the plan API over the
// plan's level-ordered copy (FP64, FP32 + FP64 refinement, 1-32 RHS).
#include <cstring>

#include "internal.h"
#include "plan.h"
#include "solve_kernels.cuh"

namespace sptrsv {

namespace {

constexpr int kBlock = 256;
constexpr int kWarpsPerBlock = kBlock / 32;

// tile lanes of the reference's simple solver from nnz/n (solve_csr_simple.cu:121-137)
int simple_lanes(int nnz, int n)
{
    int average = n > 0 ? nnz / n : 0;
    if (average <= 2) return 2;
    if (average <= 5) return 4;
    if (average <= 11) return 8;
    if (average <= 23) return 16;
    return 32;
}

bool pow2_lanes(int l) { return l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32; }

int grid_for(long long work, int block)
{
    long long g = (work + block - 1) / block;
    long long cap = (long long)ctx()->num_sms * 16;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

// Reference-named solves over the caller's CSR.  lanes = 0 picks the
// reference's choice (simple: by nnz/n; order: 32).
int solve_reference(sp_mat_t* mat, dfr_analysis_info_t* info, const double* b, double* x, int n, MODE mode,
                    int lanes, cudaStream_t s)
{
    if (!mat || !b || !x || n != mat->nr || n < 0) return set_error(SPTRSV_ERR_INVALID_ARG, "solve: bad arguments");
    if (n == 0) return ok();
    Ctx* c = ctx();
    if (!c) return set_error(SPTRSV_ERR_CUDA, "solve: no CUDA device");
    if (mode != SIMPLE && (!info || !info->iorder))
        return set_error(SPTRSV_ERR_NOT_ANALYSED, "solve: ORDER/MULTIROW need an analysis");
    if (lanes && !pow2_lanes(lanes)) return set_error(SPTRSV_ERR_INVALID_ARG, "solve: lanes must be 1,2,4,8,16,32");
    SPT_CUDA(cudaMemsetAsync(x, 0xFF, sizeof(double) * (size_t)n, s));
    NatMat m{mat->ia, mat->ja, mat->a, mode == SIMPLE ? nullptr : info->iorder};
    auto kern = k_sptrsv<NatMat, double, double, OUT_X>;
    const unsigned long long budget = wait_budget_ns();
    if (mode == MULTIROW) {
        const int* ibase = info->ibase_row;
        const int* ivect = info->ivect_size_warp;
        int nw = info->n_warps;
        if (!ibase) {  // analysed in ORDER mode: use the map kept with the analysis
            AnalysisRec* rec = find_analysis(info->row_ctr);
            if (!rec) return set_error(SPTRSV_ERR_NOT_ANALYSED, "solve: no multirow map for this analysis");
            ibase = rec->d_ibase;
            ivect = rec->d_ivect;
            nw = rec->n_warps;
        }
        SPT_CUDA(launch_persistent(kern, kBlock, 0, div_up(nw, kWarpsPerBlock), s, m, n, nw, 0, ibase, ivect, b, x,
                                   (double*)nullptr, c->d_status, budget));
    } else {
        int L = lanes ? lanes : (mode == SIMPLE ? simple_lanes(mat->nnz, n) : 32);
        int ntasks = div_up(n, 32 / L);
        SPT_CUDA(launch_persistent(kern, kBlock, 0, div_up(ntasks, kWarpsPerBlock), s, m, n, ntasks, L,
                                   (const int*)nullptr, (const int*)nullptr, b, x, (double*)nullptr, c->d_status,
                                   budget));
    }
    return ok();
}

// ---- plan ----------------------------------------------------------------------

namespace {

__global__ void k_plan_rows(const int* __restrict__ rowptr, const int* __restrict__ iorder, int n,
                            int* __restrict__ len, int* __restrict__ rowid)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x) {
        if (k == n) {
            len[k] = 0;
            continue;
        }
        int r = iorder[k];
        rowid[k] = r;
        len[k] = rowptr[r + 1] - rowptr[r] - 1;
    }
}

// one warp per position copies the row's off-diagonal entries and diagonal
__global__ void k_plan_fill(const int* __restrict__ rowptr, const int* __restrict__ col, const double* __restrict__ val,
                            const int* __restrict__ rowid, const int* __restrict__ ptr, int n, int* __restrict__ pcol,
                            double* __restrict__ pval, float* __restrict__ pval32, double* __restrict__ dg,
                            float* __restrict__ dg32)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long k = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nw) {
        int r = rowid[k];
        int s = rowptr[r], e = rowptr[r + 1] - 1, o = ptr[k];
        for (int p = s + lane; p < e; p += 32) {
            double v = val[p];
            pcol[o + p - s] = col[p];
            if (pval) pval[o + p - s] = v;
            pval32[o + p - s] = (float)v;
        }
        if (lane == 0) {
            dg[k] = val[e];
            dg32[k] = (float)val[e];
        }
    }
}

template <typename T>
cudaError_t dalloc(T** p, long long count)
{
    if (count < 1) count = 1;
    return cudaMalloc((void**)p, sizeof(T) * (size_t)count);
}

void plan_free_arrays(sptrsv_plan_s* p)
{
    cudaFree(p->ptr); cudaFree(p->rowid); cudaFree(p->col); cudaFree(p->val64); cudaFree(p->val32);
    cudaFree(p->dg64); cudaFree(p->dg32); cudaFree(p->inv); cudaFree(p->ibase); cudaFree(p->ivect);
    cudaFree(p->w32a); cudaFree(p->w32b); cudaFree(p->hb); cudaFree(p->hx);
}

}  // namespace

int plan_fill_values(sptrsv_plan_s* p, const sp_mat_t* L, cudaStream_t s)
{
    if (p->n == 0) return 0;
    k_plan_fill<<<grid_for((long long)p->n * 32, kBlock), kBlock, 0, s>>>(L->ia, L->ja, L->a, p->rowid, p->ptr, p->n,
                                                                          p->col, p->val64, p->val32, p->dg64, p->dg32);
    SPT_CUDA(cudaGetLastError());
    return 0;
}

int plan_ensure_work(sptrsv_plan_s* p, int nrhs)
{
    if (nrhs <= p->cap_rhs) return 0;
    cudaFree(p->w32a);
    cudaFree(p->w32b);
    p->w32a = p->w32b = nullptr;
    p->cap_rhs = 0;
    SPT_CUDA(dalloc(&p->w32a, (long long)p->n * nrhs));
    SPT_CUDA(dalloc(&p->w32b, (long long)p->n * nrhs));
    p->cap_rhs = nrhs;
    return 0;
}

// Launch one sync-free solve over the plan layout.
template <typename V, typename T, typename BT, int OUT>
int plan_launch(sptrsv_plan_s* p, const V* val, const V* dg, const BT* b, T* x, double* x64, int nrhs, cudaStream_t s)
{
    Ctx* c = ctx();
    const sptrsv_schedule_t& sc = p->sched;
    PermMat<V> m{p->ptr, p->rowid, p->col, val, dg, sc.variant == SPTRSV_VAR_SIMPLE ? p->inv : nullptr};
    const unsigned long long budget = wait_budget_ns();
    const int n = p->n;
    if (nrhs > 1) {
        int kp = 1;
        while (kp < nrhs) kp <<= 1;
        int ntasks = div_up(n, 32 / kp);
        auto kern = k_sptrsv_mrhs<PermMat<V>, T, BT, OUT>;
        SPT_CUDA(launch_persistent(kern, kBlock, 0, div_up(ntasks, kWarpsPerBlock), s, m, n, nrhs, kp, b, x, x64,
                                   c->d_status, budget));
        return 0;
    }
    auto kern = k_sptrsv<PermMat<V>, T, BT, OUT>;
    if (sc.variant == SPTRSV_VAR_MULTIROW) {
        SPT_CUDA(launch_persistent(kern, kBlock, 0, div_up(p->n_warps, kWarpsPerBlock), s, m, n, p->n_warps, 0,
                                   (const int*)p->ibase, (const int*)p->ivect, b, x, x64, c->d_status, budget));
    } else {
        int L = 32 / sc.rows_per_warp;
        int ntasks = div_up(n, sc.rows_per_warp);
        SPT_CUDA(launch_persistent(kern, kBlock, 0, div_up(ntasks, kWarpsPerBlock), s, m, n, ntasks, L,
                                   (const int*)nullptr, (const int*)nullptr, b, x, x64, c->d_status, budget));
    }
    return 0;
}

int plan_residual(sptrsv_plan_s* p, const double* b, const double* x, float* r32, double* r64, int nrhs,
                  cudaStream_t s)
{
    PermMat<double> m{p->ptr, p->rowid, p->col, p->val64, p->dg64, nullptr};
    const int n = p->n;
    if (nrhs > 1) {
        int kp = 1;
        while (kp < nrhs) kp <<= 1;
        long long work = (long long)div_up(n, 32 / kp) * 32;
        if (r32) k_residual_mrhs<float><<<grid_for(work, kBlock), kBlock, 0, s>>>(m, n, nrhs, kp, b, x, r32);
        else k_residual_mrhs<double><<<grid_for(work, kBlock), kBlock, 0, s>>>(m, n, nrhs, kp, b, x, r64);
    } else {
        int avg = n > 0 ? p->nnz_off / n : 0;
        int L = avg <= 1 ? 1 : avg <= 2 ? 2 : avg <= 4 ? 4 : avg <= 8 ? 8 : avg <= 16 ? 16 : 32;
        long long work = (long long)div_up(n, 32 / L) * 32;
        if (r32) k_residual<float><<<grid_for(work, kBlock), kBlock, 0, s>>>(m, n, L, b, x, r32);
        else k_residual<double><<<grid_for(work, kBlock), kBlock, 0, s>>>(m, n, L, b, x, r64);
    }
    SPT_CUDA(cudaGetLastError());
    return 0;
}

int plan_solve_f64(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s)
{
    SPT_CUDA(cudaMemsetAsync(x, 0xFF, sizeof(double) * (size_t)p->n * nrhs, s));
    return plan_launch<double, double, double, OUT_X>(p, p->val64, p->dg64, b, x, nullptr, nrhs, s);
}

int plan_solve_ir(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s)
{
    int e = plan_ensure_work(p, nrhs);
    if (e) return e;
    const size_t bytes32 = sizeof(float) * (size_t)p->n * nrhs;
    SPT_CUDA(cudaMemsetAsync(p->w32a, 0xFF, bytes32, s));
    e = plan_launch<float, float, double, OUT_SET64>(p, p->val32, p->dg32, b, p->w32a, x, nrhs, s);
    if (e) return e;
    for (int it = 0; it < p->sched.ir_max_iters; it++) {
        e = plan_residual(p, b, x, p->w32b, nullptr, nrhs, s);
        if (e) return e;
        SPT_CUDA(cudaMemsetAsync(p->w32a, 0xFF, bytes32, s));
        e = plan_launch<float, float, float, OUT_ADD64>(p, p->val32, p->dg32, p->w32b, p->w32a, x, nrhs, s);
        if (e) return e;
    }
    return 0;
}

}  // namespace sptrsv

using namespace sptrsv;

extern "C" {

void csr_L_solve_simple(sp_mat_t* mat, const VALUE_TYPE* b, VALUE_TYPE* x, int n, int* is_solved)
{
    (void)is_solved;
    solve_reference(mat, nullptr, b, x, n, SIMPLE, 0, 0);
}

void csr_L_solve_order(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b, VALUE_TYPE* x, int n,
                       cudaStream_t stream)
{
    solve_reference(mat, info, b, x, n, ORDER, 32, stream);
}

void csr_L_solve_multirow(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b, VALUE_TYPE* x, int n,
                          cudaStream_t stream)
{
    solve_reference(mat, info, b, x, n, MULTIROW, 0, stream);
}

int sptrsv_solve_order_tile(sp_mat_t* mat, dfr_analysis_info_t* info, const double* b, double* x, int tile,
                            cudaStream_t stream)
{
    if (!pow2_lanes(tile)) return set_error(SPTRSV_ERR_INVALID_ARG, "order_tile: tile must be 1,2,4,8,16,32");
    return solve_reference(mat, info, b, x, mat ? mat->nr : -1, ORDER, tile, stream);
}

int sptrsv_plan_create(const sp_mat_t* L, const dfr_analysis_info_t* info, sptrsv_plan_t* out)
{
    if (!L || !info || !out) return set_error(SPTRSV_ERR_INVALID_ARG, "plan_create: NULL argument");
    *out = nullptr;
    AnalysisRec* rec = find_analysis(info->row_ctr);
    if (!rec || !info->iorder || rec->n != L->nr)
        return set_error(SPTRSV_ERR_NOT_ANALYSED, "plan_create: info is not an analysis of this matrix");
    Ctx* c = ctx();
    if (!c) return set_error(SPTRSV_ERR_CUDA, "plan_create: no CUDA device");
    cudaStream_t s = 0;
    sptrsv_plan_s* p = new sptrsv_plan_s();
    p->device = c->device;
    p->n = L->nr;
    p->nnz_off = L->nnz - L->nr;
    p->nlevs = rec->nlevs;
    p->n_warps = rec->n_warps;
    const int n = p->n;
    int* d_scr = nullptr;
    auto fail = [&](int code) {
        cudaFree(d_scr);
        plan_free_arrays(p);
        delete p;
        return code;
    };
#define PCHK(call)                                                \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, #call)); \
    } while (0)
    PCHK(dalloc(&p->ptr, (long long)n + 1));
    PCHK(dalloc(&p->rowid, n));
    PCHK(dalloc(&p->col, p->nnz_off));
    PCHK(dalloc(&p->val64, p->nnz_off));
    PCHK(dalloc(&p->val32, p->nnz_off));
    PCHK(dalloc(&p->dg64, n));
    PCHK(dalloc(&p->dg32, n));
    PCHK(dalloc(&p->inv, n));
    PCHK(dalloc(&p->ibase, (long long)p->n_warps + 1));
    PCHK(dalloc(&p->ivect, p->n_warps));
    PCHK(dalloc(&d_scr, scan_scratch_ints((long long)n + 1)));
    if (n > 0) {
        k_plan_rows<<<grid_for((long long)n + 1, kBlock), kBlock, 0, s>>>(L->ia, info->iorder, n, p->ptr, p->rowid);
        PCHK(cudaGetLastError());
        PCHK(scan_exclusive(p->ptr, p->ptr, (long long)n + 1, d_scr, s));
        int e = plan_fill_values(p, L, s);
        if (e) return fail(e);
        PCHK(cudaMemcpyAsync(p->inv, info->inv_iorder, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    }
    PCHK(cudaMemcpyAsync(p->ibase, rec->d_ibase, sizeof(int) * ((size_t)p->n_warps + 1), cudaMemcpyDeviceToDevice, s));
    if (p->n_warps > 0)
        PCHK(cudaMemcpyAsync(p->ivect, rec->d_ivect, sizeof(int) * (size_t)p->n_warps, cudaMemcpyDeviceToDevice, s));
    PCHK(cudaStreamSynchronize(s));
#undef PCHK
    cudaFree(d_scr);
    p->sched.variant = SPTRSV_VAR_MULTIROW;
    p->sched.rows_per_warp = 1;
    p->sched.block_warps = kWarpsPerBlock;
    p->sched.ir_max_iters = 2;
    *out = p;
    return ok();
}

int sptrsv_plan_destroy(sptrsv_plan_t p)
{
    if (!p) return ok();
    plan_free_arrays(p);
    delete p;
    return ok();
}

int sptrsv_plan_set_schedule(sptrsv_plan_t p, const sptrsv_schedule_t* s)
{
    if (!p || !s) return set_error(SPTRSV_ERR_INVALID_ARG, "set_schedule: NULL argument");
    if (s->variant < 0 || s->variant >= SPTRSV_N_VARIANTS || s->variant == SPTRSV_VAR_CLUSTER)
        return set_error(SPTRSV_ERR_UNSUPPORTED, "set_schedule: variant %d not available", s->variant);
    if (!pow2_lanes(s->rows_per_warp)) return set_error(SPTRSV_ERR_INVALID_ARG, "set_schedule: rows_per_warp");
    if (s->ir_max_iters < 0 || s->ir_max_iters > 16) return set_error(SPTRSV_ERR_INVALID_ARG, "set_schedule: ir_max_iters");
    p->sched = *s;
    p->sched.block_warps = kWarpsPerBlock;
    return ok();
}

int sptrsv_plan_get_schedule(sptrsv_plan_t p, sptrsv_schedule_t* s)
{
    if (!p || !s) return set_error(SPTRSV_ERR_INVALID_ARG, "get_schedule: NULL argument");
    *s = p->sched;
    return ok();
}

int sptrsv_plan_update_values(sptrsv_plan_t p, const sp_mat_t* L)
{
    if (!p || !L || L->nr != p->n || L->nnz - L->nr != p->nnz_off)
        return set_error(SPTRSV_ERR_INVALID_ARG, "update_values: matrix does not match the plan");
    int e = plan_fill_values(p, L, 0);
    if (e) return e;
    SPT_CUDA(cudaStreamSynchronize(0));
    return ok();
}

int sptrsv_solve_f64(sptrsv_plan_t p, const double* b, double* x, int nrhs, cudaStream_t stream)
{
    if (!p || !b || !x || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "solve_f64: bad arguments");
    if (p->n == 0) return ok();
    int e = plan_solve_f64(p, b, x, nrhs, stream);
    return e ? e : ok();
}

int sptrsv_solve_ir(sptrsv_plan_t p, const double* b, double* x, int nrhs, cudaStream_t stream)
{
    if (!p || !b || !x || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "solve_ir: bad arguments");
    if (p->n == 0) return ok();
    int e = plan_solve_ir(p, b, x, nrhs, stream);
    return e ? e : ok();
}

int sptrsv_solve_f32(sptrsv_plan_t p, const double* b, float* x32, int nrhs, cudaStream_t stream)
{
    if (!p || !b || !x32 || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "solve_f32: bad arguments");
    if (p->n == 0) return ok();
    SPT_CUDA(cudaMemsetAsync(x32, 0xFF, sizeof(float) * (size_t)p->n * nrhs, stream));
    int e = plan_launch<float, float, double, OUT_X>(p, p->val32, p->dg32, b, x32, nullptr, nrhs, stream);
    return e ? e : ok();
}

int sptrsv_residual_f64(sptrsv_plan_t p, const double* b, const double* x, double* r, int nrhs, cudaStream_t stream)
{
    if (!p || !b || !x || !r || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "residual: bad arguments");
    if (p->n == 0) return ok();
    int e = plan_residual(p, b, x, nullptr, r, nrhs, stream);
    return e ? e : ok();
}

int sptrsv_solve_host(sptrsv_plan_t p, const double* hb, double* hx, int nrhs, int precision, cudaStream_t s)
{
    if (!p || !hb || !hx || nrhs < 1 || nrhs > 32 || (precision != 32 && precision != 64))
        return set_error(SPTRSV_ERR_INVALID_ARG, "solve_host: bad arguments");
    if (p->n == 0) return ok();
    const size_t bytes = sizeof(double) * (size_t)p->n * nrhs;
    if (nrhs > p->cap_host) {
        cudaFree(p->hb);
        cudaFree(p->hx);
        p->hb = p->hx = nullptr;
        p->cap_host = 0;
        SPT_CUDA(cudaMalloc((void**)&p->hb, bytes));
        SPT_CUDA(cudaMalloc((void**)&p->hx, bytes));
        p->cap_host = nrhs;
    }
    SPT_CUDA(cudaMemcpyAsync(p->hb, hb, bytes, cudaMemcpyHostToDevice, s));
    int e = precision == 32 ? plan_solve_ir(p, p->hb, p->hx, nrhs, s) : plan_solve_f64(p, p->hb, p->hx, nrhs, s);
    if (e) return e;
    SPT_CUDA(cudaMemcpyAsync(hx, p->hx, bytes, cudaMemcpyDeviceToHost, s));
    e = sync_status(s);
    return e ? e : ok();
}

}  // extern "C"
