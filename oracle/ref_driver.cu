/*
 * ref_driver.cu — a small C-ABI driver around the reference's own CUDA
 * kernels (HCL-Fing/SPTRSV analysis/analysis_csr.cu and
 * solver/solve_csr_{simple,order,multirow}.cu, compiled unmodified from the
 * reference tree by oracle/Makefile into oracle/_ref/libsptrsv_ref.so).
 *
 * TEST INFRASTRUCTURE ONLY: it produces the reference's own analysis arrays
 * and solutions on a GPU so that the CPU oracle and the library can be
 * checked against them, and it times the reference kernels as a comparator.
 *
 * The reference's interface.cu does not compile (its definitions disagree
 * with header/interface.h), so this driver replaces it: it fills a
 * caller-side dfr_analysis_info_t and calls multirow_analysis_base_GPU and
 * the csr_L_solve_* functions directly, the flow interface.cu:28-95 intends.
 *
 * Memory safety: the matrix arrays handed to the reference are padded
 * (rowptr gets an extra entry equal to nnz; colidx and values get 64 spare
 * zero entries) because its kernels read col_idx[row_ptr[i]+lane] before the
 * loop bound check (analysis_csr.cu:145) and row_ptr[n+1] for the tile with
 * groupId == n (:127,:133).  Its own allocations get slack from ref_shim.h.
 * Every call runs under a host watchdog thread that ends the process if the
 * reference does not return in time (its device waits are unbounded,
 * analysis_csr.cu:150, solve_csr_order.cu:254, solve_csr_multirow.cu:84).
 */
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <unistd.h>
#include <vector>
#include <algorithm>

#include "common.h"
#include "dfr_syncfree.h"

/* Reference entry points (header/analysis.h:20, header/solver.h:5-7). */
void multirow_analysis_base_GPU(dfr_analysis_info_t** info, sp_mat_t* gpu_L, MODE mode);
void csr_L_solve_simple(sp_mat_t* mat, const VALUE_TYPE* b, VALUE_TYPE* x, int n, int* is_solved);
void csr_L_solve_order(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b, VALUE_TYPE* x,
                       int n, cudaStream_t stream);
void csr_L_solve_multirow(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b, VALUE_TYPE* x,
                          int n, cudaStream_t stream);

#define REF_SHIM_PAD 4096

static std::mutex g_alloc_mu;
static bool g_capture = false;
static std::vector<std::pair<void*, size_t>> g_allocs;

extern "C" cudaError_t ref_shim_cudaMalloc(void** p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes + REF_SHIM_PAD);
    if (e == cudaSuccess) {
        cudaMemset((char*)*p + bytes, 0, REF_SHIM_PAD);
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        if (g_capture) g_allocs.push_back({*p, bytes});
    }
    return e;
}

/* ---- watchdog: ends the process if a reference call does not return ---- */
static std::mutex g_wd_mu;
static std::condition_variable g_wd_cv;
static bool g_wd_armed = false;
static double g_wd_seconds = 60.0;
static const char* g_wd_what = "";

struct Watchdog {
    std::thread th;
    explicit Watchdog(const char* what)
    {
        std::unique_lock<std::mutex> lk(g_wd_mu);
        g_wd_armed = true;
        g_wd_what = what;
        double secs = g_wd_seconds;
        lk.unlock();
        th = std::thread([secs]() {
            std::unique_lock<std::mutex> l2(g_wd_mu);
            bool done = g_wd_cv.wait_for(l2, std::chrono::duration<double>(secs), [] { return !g_wd_armed; });
            if (!done) {
                fprintf(stderr, "ref_driver: reference call '%s' did not return within %.1f s; exiting\n",
                        g_wd_what, secs);
                fflush(stderr);
                _exit(3);
            }
        });
    }
    ~Watchdog()
    {
        {
            std::lock_guard<std::mutex> lk(g_wd_mu);
            g_wd_armed = false;
        }
        g_wd_cv.notify_all();
        th.join();
    }
};

extern "C" void ref_set_watchdog_seconds(double s) { g_wd_seconds = s; }

/* ---- padded device copy of a host CSR ---- */
struct DevCsr {
    sp_mat_t m{};
};

static int upload(int n, const int* rowptr, const int* colidx, const double* val, DevCsr* d)
{
    int nnz = rowptr[n] - rowptr[0];
    std::vector<int> rp(rowptr, rowptr + n + 1);
    rp.push_back(rp[n]);
    std::vector<int> ci(colidx, colidx + nnz);
    ci.resize((size_t)nnz + 64, 0);
    // values in the build's VALUE_TYPE (double, the reference's Makefile:7)
    std::vector<VALUE_TYPE> va((size_t)nnz + 64, (VALUE_TYPE)0);
    if (val) std::transform(val, val + nnz, va.begin(), [](double v) { return (VALUE_TYPE)v; });
    else std::fill(va.begin(), va.begin() + nnz, (VALUE_TYPE)1);
    if (cudaMalloc((void**)&d->m.ia, sizeof(int) * (n + 2)) != cudaSuccess) return -4;
    if (cudaMalloc((void**)&d->m.ja, sizeof(int) * ci.size()) != cudaSuccess) return -4;
    if (cudaMalloc((void**)&d->m.a, sizeof(VALUE_TYPE) * va.size()) != cudaSuccess) return -4;
    cudaMemcpy(d->m.ia, rp.data(), sizeof(int) * (n + 2), cudaMemcpyHostToDevice);
    cudaMemcpy(d->m.ja, ci.data(), sizeof(int) * ci.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d->m.a, va.data(), sizeof(VALUE_TYPE) * va.size(), cudaMemcpyHostToDevice);
    d->m.nr = n;
    d->m.nc = n;
    d->m.nnz = nnz;
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

static void release(DevCsr* d)
{
    cudaFree(d->m.ia);
    cudaFree(d->m.ja);
    cudaFree(d->m.a);
}

static void release_info(dfr_analysis_info_t* info)
{
    cudaFree(info->iorder);
    cudaFree(info->row_ctr);
    if (info->mode == MULTIROW || info->mode == ALL) {
        cudaFree(info->ibase_row);
        cudaFree(info->ivect_size_warp);
    }
}

/* Runs the reference analysis on a host CSR and copies its results back.
 * mode: 1 ORDER, 2 MULTIROW.  Output buffers: levels[n] (the level array the
 * reference computes, read from its first allocation), iorder[n],
 * ibase_row[n+1], ivect[n] (n_warps <= n always).  Returns 0 or < 0. */
extern "C" int ref_analysis(int n, const int* rowptr, const int* colidx, int mode, int* nlevs,
                            int* n_warps, int* levels, int* iorder, int* ibase_row, int* ivect)
{
    DevCsr d;
    if (upload(n, rowptr, colidx, nullptr, &d)) return -4;
    dfr_analysis_info_t info_s;
    memset(&info_s, 0, sizeof(info_s));
    info_s.mode = (MODE)mode;
    dfr_analysis_info_t* info = &info_s;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        g_allocs.clear();
        g_capture = true;
    }
    {
        Watchdog wd("multirow_analysis_base_GPU");
        multirow_analysis_base_GPU(&info, &d.m, (MODE)mode);
        cudaDeviceSynchronize();
    }
    void* lev_ptr = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        g_capture = false;
        if (!g_allocs.empty() && g_allocs[0].second == sizeof(int) * (size_t)n) lev_ptr = g_allocs[0].first;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "ref_analysis: %s\n", cudaGetErrorString(e));
        return -4;
    }
    *nlevs = info->nlevs;
    *n_warps = (mode == MULTIROW || mode == ALL) ? info->n_warps : 0;
    if (levels) {
        if (!lev_ptr) return -6;
        cudaMemcpy(levels, lev_ptr, sizeof(int) * n, cudaMemcpyDeviceToHost);
    }
    cudaMemcpy(iorder, info->iorder, sizeof(int) * n, cudaMemcpyDeviceToHost);
    if (mode == MULTIROW || mode == ALL) {
        cudaMemcpy(ibase_row, info->ibase_row, sizeof(int) * (info->n_warps + 1), cudaMemcpyDeviceToHost);
        cudaMemcpy(ivect, info->ivect_size_warp, sizeof(int) * info->n_warps, cudaMemcpyDeviceToHost);
    }
    release_info(info);
    release(&d);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

/* Solves L x = b with a reference solver (variant 0 simple, 1 order,
 * 2 multirow) on host arrays; runs `reps` timed solves (CUDA events around
 * the reference solve call, which includes its own memsets, the reference's
 * timing scope in header/common.h:103-124) and returns the median ms in
 * *ms_median (may be NULL).  x receives the last solve's result. */
extern "C" int ref_solve(int variant, int n, const int* rowptr, const int* colidx, const double* val,
                         const double* b, double* x, int reps, float* ms_median)
{
    DevCsr d;
    if (upload(n, rowptr, colidx, val, &d)) return -4;
    dfr_analysis_info_t info_s;
    memset(&info_s, 0, sizeof(info_s));
    dfr_analysis_info_t* info = &info_s;
    if (variant != 0) {
        info_s.mode = variant == 1 ? ORDER : MULTIROW;
        Watchdog wd("multirow_analysis_base_GPU");
        multirow_analysis_base_GPU(&info, &d.m, info_s.mode);
        cudaDeviceSynchronize();
    }
    VALUE_TYPE *d_b = nullptr, *d_x = nullptr;
    int* is_solved = nullptr;
    cudaMalloc((void**)&d_b, sizeof(VALUE_TYPE) * (n + 64));
    cudaMalloc((void**)&d_x, sizeof(VALUE_TYPE) * (n + 64));
    cudaMalloc((void**)&is_solved, sizeof(int) * (n + 64));
    {
        std::vector<VALUE_TYPE> hb(b, b + n);
        cudaMemcpy(d_b, hb.data(), sizeof(VALUE_TYPE) * n, cudaMemcpyHostToDevice);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> ts;
    if (reps < 1) reps = 1;
    for (int r = 0; r < reps; r++) {
        cudaMemset(d_x, 0, sizeof(VALUE_TYPE) * n);
        Watchdog wd(variant == 0 ? "csr_L_solve_simple" : variant == 1 ? "csr_L_solve_order" : "csr_L_solve_multirow");
        cudaEventRecord(e0, 0);
        if (variant == 0) csr_L_solve_simple(&d.m, d_b, d_x, n, is_solved);
        else if (variant == 1) csr_L_solve_order(&d.m, info, d_b, d_x, n, 0);
        else csr_L_solve_multirow(&d.m, info, d_b, d_x, n, 0);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        ts.push_back(ms);
    }
    cudaError_t e = cudaGetLastError();
    {
        std::vector<VALUE_TYPE> hx(n);
        cudaMemcpy(hx.data(), d_x, sizeof(VALUE_TYPE) * n, cudaMemcpyDeviceToHost);
        std::copy(hx.begin(), hx.end(), x);
    }
    std::sort(ts.begin(), ts.end());
    if (ms_median) *ms_median = ts[ts.size() / 2];
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_b);
    cudaFree(d_x);
    cudaFree(is_solved);
    if (variant != 0) release_info(info);
    release(&d);
    if (e != cudaSuccess) {
        fprintf(stderr, "ref_solve: %s\n", cudaGetErrorString(e));
        return -4;
    }
    return 0;
}
