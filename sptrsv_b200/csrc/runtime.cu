// runtime.cu — per-device context, error reporting, the analysis registry
// and the reference interface (header/interface.h:6-9, header/analysis.h:20).
//
// The reference's interface.cu does not compile and loses its results
// (allocate_memory assigns its out-parameter locally, interface.cu:10;
// run_solver mallocs x internally, :43).  This implementation follows the
// header prototypes: caller-allocated structs, library-owned device arrays,
// results written to the caller's buffers.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace sptrsv {

// ---- errors ----------------------------------------------------------------
static thread_local int t_err = SPTRSV_OK;
static thread_local char t_msg[512] = "ok";

int set_error(int code, const char* fmt, ...)
{
    t_err = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof(t_msg), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
    return set_error(SPTRSV_ERR_CUDA, "CUDA error %s (%s) in %s", cudaGetErrorName(e), cudaGetErrorString(e), where);
}

// ---- context -----------------------------------------------------------------
static std::mutex g_ctx_mu;
static std::vector<Ctx*> g_ctx;
static unsigned long long g_budget_ns = 2000000000ULL;

Ctx* ctx()
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return nullptr;
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if ((int)g_ctx.size() <= dev) g_ctx.resize(dev + 1, nullptr);
    if (!g_ctx[dev]) {
        Ctx* c = new Ctx();
        c->device = dev;
        cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaMalloc((void**)&c->d_status, sizeof(DevStatus)) != cudaSuccess) {
            delete c;
            return nullptr;
        }
        cudaMemset(c->d_status, 0, sizeof(DevStatus));
        cudaDeviceSynchronize();
        g_ctx[dev] = c;
    }
    return g_ctx[dev];
}

unsigned long long wait_budget_ns() { return g_budget_ns; }

int grid_for(long long work, int block)
{
    long long g = (work + block - 1) / block;
    long long cap = (long long)ctx()->num_sms * 16;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

int sync_status(cudaStream_t stream)
{
    Ctx* c = ctx();
    if (!c) return set_error(SPTRSV_ERR_CUDA, "no CUDA device");
    DevStatus h{};
    SPT_CUDA(cudaStreamSynchronize(stream));
    SPT_CUDA(cudaMemcpy(&h, c->d_status, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.code != 0) {
        DevStatus z{};
        SPT_CUDA(cudaMemcpy(c->d_status, &z, sizeof(z), cudaMemcpyHostToDevice));
        if (h.code == SPTRSV_ERR_TIMEOUT)
            return set_error(SPTRSV_ERR_TIMEOUT, "device wait ran out of budget at row %d", h.row);
        return set_error(h.code, "device error %d at row %d", h.code, h.row);
    }
    return SPTRSV_OK;
}

// ---- analysis registry ---------------------------------------------------------
static std::mutex g_reg_mu;
static std::unordered_map<const int*, AnalysisRec*> g_reg;

void register_analysis(const int* key, AnalysisRec* rec)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_reg[key] = rec;
}
AnalysisRec* find_analysis(const int* key)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    auto it = g_reg.find(key);
    return it == g_reg.end() ? nullptr : it->second;
}
AnalysisRec* unregister_analysis(const int* key)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    auto it = g_reg.find(key);
    if (it == g_reg.end()) return nullptr;
    AnalysisRec* r = it->second;
    g_reg.erase(it);
    return r;
}

// One thread waits on a word that nothing writes; the bounded wait must end
// with SPTRSV_ERR_TIMEOUT in the status block and the kernel must return.
__global__ void k_wait_unset_flag(const int* flag, DevStatus* st, unsigned long long budget)
{
    int v;
    wait_ready(flag, v, st, budget, -1);
}

int solve_reference(sp_mat_t* mat, dfr_analysis_info_t* info, const double* b, double* x, int n, MODE mode,
                    int lanes, cudaStream_t stream);

}  // namespace sptrsv

using namespace sptrsv;

extern "C" {

int sptrsv_last_error(void) { return t_err; }
const char* sptrsv_last_error_string(void) { return t_msg; }
const char* sptrsv_version(void) { return "sptrsv_b200 0.1 (sm_100a)"; }

void sptrsv_set_wait_budget_ns(unsigned long long ns) { g_budget_ns = ns ? ns : 1; }

int sptrsv_sync_status(cudaStream_t stream)
{
    return ::sptrsv::abi_guard([&]() -> int {
        int e = sync_status(stream);
        return e ? e : ok();
    });
}

int sptrsv_selftest_bounded_wait(unsigned long long budget_ns)
{
    return ::sptrsv::abi_guard([&]() -> int {
        Ctx* c = ctx();
        if (!c) return set_error(SPTRSV_ERR_CUDA, "selftest: no CUDA device");
        int e = sync_status(0);
        if (e) return e;
        int* flag = nullptr;
        SPT_CUDA(cudaMalloc((void**)&flag, sizeof(int)));
        cudaError_t ce = cudaMemset(flag, 0, sizeof(int));
        if (ce == cudaSuccess) {
            k_wait_unset_flag<<<1, 1>>>(flag, c->d_status, budget_ns);
            ce = cudaGetLastError();
        }
        e = ce == cudaSuccess ? sync_status(0) : cuda_fail(ce, "selftest launch");
        cudaFree(flag);
        return e;
    });
}

int sptrsv_check_csr_host(const int* rowptr, const int* colidx, int n, int* bad_row)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (bad_row) *bad_row = -1;
        if (n < 0 || (n > 0 && (!rowptr || !colidx))) return set_error(SPTRSV_ERR_INVALID_ARG, "check_csr: bad arguments");
        if (n > 0 && rowptr[0] != 0) {
            if (bad_row) *bad_row = 0;
            return set_error(SPTRSV_ERR_INVALID_CSR, "check_csr: rowptr[0] != 0");
        }
        for (int i = 0; i < n; i++) {
            int s = rowptr[i], e = rowptr[i + 1];
            bool bad = e <= s || colidx[e - 1] != i;
            for (int p = s; p < e - 1 && !bad; p++)
                if (colidx[p] < 0 || colidx[p] >= i || (p > s && colidx[p] <= colidx[p - 1])) bad = true;
            if (bad) {
                if (bad_row) *bad_row = i;
                return set_error(SPTRSV_ERR_INVALID_CSR, "check_csr: row %d is not lower-triangular CSR with sorted "
                                 "columns and the diagonal last", i);
            }
        }
        return ok();
    });
}

// header/interface.h:6 — host CSR to device.
int allocate_memory(int* csrRowPtrL, int* csrColIdxL, VALUE_TYPE* csrValL, int n, sp_mat_t* gpu_L, MODE mode)
{
    return ::sptrsv::abi_guard([&]() -> int {
        (void)mode;
        if (!gpu_L || n < 0 || (n > 0 && (!csrRowPtrL || !csrColIdxL || !csrValL)))
            return set_error(SPTRSV_ERR_INVALID_ARG, "allocate_memory: bad arguments");
        int bad = -1;
        int e = sptrsv_check_csr_host(csrRowPtrL, csrColIdxL, n, &bad);
        if (e) return e;
        if (!ctx()) return set_error(SPTRSV_ERR_CUDA, "allocate_memory: no CUDA device");
        int nnz = n > 0 ? csrRowPtrL[n] - csrRowPtrL[0] : 0;
        memset(gpu_L, 0, sizeof(*gpu_L));
        SPT_CUDA(cudaMalloc((void**)&gpu_L->ia, sizeof(int) * (size_t)(n + 1)));
        SPT_CUDA(cudaMalloc((void**)&gpu_L->ja, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)));
        SPT_CUDA(cudaMalloc((void**)&gpu_L->a, sizeof(double) * (size_t)(nnz > 0 ? nnz : 1)));
        SPT_CUDA(cudaMemcpy(gpu_L->ia, csrRowPtrL, sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice));
        if (nnz > 0) {
            SPT_CUDA(cudaMemcpy(gpu_L->ja, csrColIdxL, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice));
            SPT_CUDA(cudaMemcpy(gpu_L->a, csrValL, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice));
        }
        gpu_L->nr = n;
        gpu_L->nc = n;
        gpu_L->nnz = nnz;
        return ok();
    });
}

// A struct that still holds an analysis made by this library (its row_ctr
// is a registered key) owns device arrays: release them before the struct
// is overwritten, so analysing into the same struct again leaks nothing.
// Anything else in the struct (a fresh or uninitialised one) is only cleared.
static void release_held_analysis(dfr_analysis_info_t* info)
{
    MODE m = info->mode;
    if (info->row_ctr && find_analysis(info->row_ctr)) free_device_analysis(nullptr, info);
    memset(info, 0, sizeof(*info));
    info->mode = m;
}

// header/interface.h:7 — analysis per info->mode.
int run_analysis(dfr_analysis_info_t* info, sp_mat_t* gpu_L)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!info || !gpu_L) return set_error(SPTRSV_ERR_INVALID_ARG, "run_analysis: NULL argument");
        if (info->mode == SIMPLE) return set_error(SPTRSV_NO_ANALYSIS, "run_analysis: SIMPLE needs no analysis");
        if (info->mode != ORDER && info->mode != MULTIROW && info->mode != ALL)
            return set_error(SPTRSV_ERR_INVALID_ARG, "run_analysis: unknown mode %d", (int)info->mode);
        MODE m = info->mode;
        release_held_analysis(info);
        info->mode = m;
        return run_analysis_impl(info, gpu_L, m);
    });
}

// header/analysis.h:20
void multirow_analysis_base_GPU(dfr_analysis_info_t** info, sp_mat_t* gpu_L, MODE mode)
{
    ::sptrsv::abi_guard_void([&] {
        if (!info || !*info) {
            set_error(SPTRSV_ERR_INVALID_ARG, "multirow_analysis_base_GPU: *info must point to a caller-allocated struct");
            return;
        }
        if (!gpu_L) {
            set_error(SPTRSV_ERR_INVALID_ARG, "multirow_analysis_base_GPU: NULL matrix");
            return;
        }
        release_held_analysis(*info);
        (*info)->mode = mode;
        run_analysis_impl(*info, gpu_L, mode);
    });
}

// header/interface.h:8 — host b, host x.
void run_solver(sp_mat_t* gpu_L, dfr_analysis_info_t* info, VALUE_TYPE* b, VALUE_TYPE* x, int n)
{
    ::sptrsv::abi_guard_void([&] {
        if (!gpu_L || !b || !x || n != gpu_L->nr) {
            set_error(SPTRSV_ERR_INVALID_ARG, "run_solver: bad arguments");
            return;
        }
        if (n == 0) {
            ok();
            return;
        }
        if (!ctx()) {
            set_error(SPTRSV_ERR_CUDA, "run_solver: no CUDA device");
            return;
        }
        MODE mode = info ? info->mode : SIMPLE;
        if (mode == ALL) mode = MULTIROW;
        double *d_b = nullptr, *d_x = nullptr;
        auto cleanup = [&]() {
            cudaFree(d_b);
            cudaFree(d_x);
        };
        if (cudaMalloc((void**)&d_b, sizeof(double) * (size_t)n) != cudaSuccess ||
            cudaMalloc((void**)&d_x, sizeof(double) * (size_t)n) != cudaSuccess) {
            cleanup();
            set_error(SPTRSV_ERR_ALLOC, "run_solver: device allocation failed");
            return;
        }
        cudaMemcpy(d_b, b, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice);
        int e = solve_reference(gpu_L, info, d_b, d_x, n, mode, 0, 0);
        if (e == 0) e = sync_status(0);
        if (e == 0) {
            cudaError_t ce = cudaMemcpy(x, d_x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost);
            if (ce != cudaSuccess) e = cuda_fail(ce, "run_solver: copy back");
        }
        cleanup();
        if (e == 0) ok();
    });
}

// header/interface.h:9 — frees every device array of both structs.
void free_device_analysis(sp_mat_t* gpu_L, dfr_analysis_info_t* info)
{
    ::sptrsv::abi_guard_void([&] {
        if (info) {
            AnalysisRec* rec = info->row_ctr ? unregister_analysis(info->row_ctr) : nullptr;
            cudaFree(info->iorder);
            cudaFree(info->row_ctr);
            cudaFree(info->lev_size);
            cudaFree(info->inv_iorder);
            if (rec) {
                cudaFree(rec->d_levels);
                cudaFree(rec->d_counts);
                cudaFree(rec->d_ibase);
                cudaFree(rec->d_ivect);
                cudaFree(rec->d_wlev);
                for (int j = 0; j < 6; j++) cudaFree(rec->tile_tasks[j]);
                delete rec;
            } else {
                cudaFree(info->ibase_row);
                cudaFree(info->ivect_size_warp);
                cudaFree(info->warp_lev);
            }
            MODE m = info->mode;
            memset(info, 0, sizeof(*info));
            info->mode = m;
        }
        if (gpu_L) {
            cudaFree(gpu_L->ia);
            cudaFree(gpu_L->ja);
            cudaFree(gpu_L->a);
            memset(gpu_L, 0, sizeof(*gpu_L));
        }
        ok();
    });
}

int sptrsv_analysis_levels(const dfr_analysis_info_t* info, int* host_levels)
{
    return ::sptrsv::abi_guard([&]() -> int {
        AnalysisRec* rec = info ? find_analysis(info->row_ctr) : nullptr;
        if (!rec || !host_levels) return set_error(SPTRSV_ERR_NOT_ANALYSED, "analysis_levels: no analysis for this info");
        if (rec->n > 0) SPT_CUDA(cudaMemcpy(host_levels, rec->d_levels, sizeof(int) * (size_t)rec->n, cudaMemcpyDeviceToHost));
        return ok();
    });
}

int sptrsv_analysis_buckets(const dfr_analysis_info_t* info, int* host_buckets)
{
    return ::sptrsv::abi_guard([&]() -> int {
        AnalysisRec* rec = info ? find_analysis(info->row_ctr) : nullptr;
        if (!rec || !host_buckets) return set_error(SPTRSV_ERR_NOT_ANALYSED, "analysis_buckets: no analysis for this info");
        if (rec->nlevs > 0)
            SPT_CUDA(cudaMemcpy(host_buckets, rec->d_counts, sizeof(int) * (size_t)rec->nlevs * 7, cudaMemcpyDeviceToHost));
        return ok();
    });
}

}  // extern "C"
