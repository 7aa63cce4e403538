// noalloc.cu — an FP32 + FP64-refinement solve that allocates nothing.
//
// Some callers cannot allocate device memory at solve time: code running
// inside a memory pool or arena that owns every byte of the device heap,
// code that must not call cudaMalloc after start-up (real-time or
// certification rules), and callers of runtimes that only hand out fixed
// buffers.  sptrsv_solve_ir_noalloc serves them: the caller passes the
// device CSR, b and x, and the solve's scratch (two FP32 work vectors and
// a status word) lives in one file-scope __device__ array of fixed size,
// which every GPU that loads this library keeps for the life of the process.
//
// The solve needs no analysis and no plan: an FP32 solve over natural-order
// chunks (the SIMPLE schedule, values read from the caller's FP64 CSR and
// rounded on the fly), then ir_iters times an FP64 residual r = b - L x and
// an FP32 correction solve with x += d in FP64.
#include <mutex>

#include "internal.h"
#include "solve_kernels.cuh"

namespace sptrsv {

namespace {

// Largest system: SPTRSV_NOALLOC_MAX_ROWS (2^20) rows -> 2 x 4 MiB FP32 work vectors.
constexpr long long kNoallocMaxRows = SPTRSV_NOALLOC_MAX_ROWS;
constexpr size_t kNoallocBytes = 2 * sizeof(float) * kNoallocMaxRows + 256;

// Scratch: [x32 | r32 | status].  In host code `g_noalloc_scratch` names a
// host-side stand-in, not device memory; the device address comes from
// cudaGetSymbolAddress, taken once per device with that device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

std::mutex g_mu;
unsigned char* g_addr[64] = {};
int g_sms[64] = {};

int scratch_address(unsigned char** out, int* sms)
{
    int dev = -1;
    SPT_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(SPTRSV_ERR_UNSUPPORTED, "noalloc: device index %d", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "noalloc: cudaGetSymbolAddress");
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_fail(e, "noalloc: SM count");
        g_addr[dev] = (unsigned char*)p;
        g_sms[dev] = n;
    }
    *out = g_addr[dev];
    *sms = g_sms[dev];
    return 0;
}

// r = b - L x over the caller's natural-order CSR (FP64), r rounded to FP32.
// The CSR is checked as it is read: a row range outside [0, nnz] or a column
// outside [0, i] records SPTRSV_ERR_INVALID_CSR and that row (or entry) is
// skipped, so no bad index is ever used.
__global__ void __launch_bounds__(256) k_residual_nat(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                      const double* __restrict__ val, int n, int nnz,
                                                      const double* __restrict__ b, const double* __restrict__ x,
                                                      float* __restrict__ r, DevStatus* st)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const int s = rowptr[i], e = rowptr[i + 1];
        if (!(s >= 0 && s < e && e <= nnz)) {
            if (lane == 0) report(st, SPTRSV_ERR_INVALID_CSR, (int)i);
            continue;
        }
        double acc = 0.0;
        for (int p = s + lane; p < e; p += 32) {
            const int c = col[p];
            if (c < 0 || c > i) {
                report(st, SPTRSV_ERR_INVALID_CSR, (int)i);
                continue;
            }
            acc += val[p] * x[c];
        }
        for (int o = 16; o >= 1; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) r[i] = (float)(b[i] - acc);
    }
}

// Chunk solve over the natural order with an explicit grid (no occupancy
// cache, no cooperative attribute bookkeeping beyond the launch itself).
template <typename BT, int OUT>
cudaError_t launch_chunk(const NatMat& m, int n, const BT* b, float* x32, double* x, DevStatus* st, int sms,
                         cudaStream_t s)
{
    auto kern = k_sptrsv_chunk<NatMat, float, BT, OUT, true>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
    if (e != cudaSuccess) return e;
    long long need = ((long long)(n + 31) / 32 + 7) / 8;
    long long grid = (long long)per_sm * sms;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, m, n, 32, b, x32, x, st, wait_budget_ns(), 0u);
}

}  // namespace

}  // namespace sptrsv

using namespace sptrsv;

extern "C" int sptrsv_solve_ir_noalloc(const sp_mat_t* L, const double* b, double* x, int ir_iters,
                                       cudaStream_t stream)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!L || !b || !x || ir_iters < 0 || ir_iters > 16 || L->nr < 0 || L->nc != L->nr || L->nnz < L->nr ||
            (L->nr > 0 && (!L->ia || !L->ja || !L->a)))
            return set_error(SPTRSV_ERR_INVALID_ARG, "solve_ir_noalloc: bad arguments");
        if ((long long)L->nr > kNoallocMaxRows)
            return set_error(SPTRSV_ERR_UNSUPPORTED,
                             "solve_ir_noalloc: n = %d exceeds the fixed scratch limit of %lld rows", L->nr,
                             kNoallocMaxRows);
        const int n = L->nr;
        if (n == 0) return ok();
        unsigned char* base = nullptr;
        int sms = 0;
        int e = scratch_address(&base, &sms);
        if (e) return e;
        float* x32 = reinterpret_cast<float*>(base);
        float* r32 = x32 + kNoallocMaxRows;
        DevStatus* st = reinterpret_cast<DevStatus*>(base + 2 * sizeof(float) * kNoallocMaxRows);
        // the array keeps the previous call's contents: reset what must start clean
        SPT_CUDA(cudaMemsetAsync(st, 0, sizeof(DevStatus), stream));
        SPT_CUDA(cudaMemsetAsync(x32, 0xFF, sizeof(float) * (size_t)n, stream));
        NatMat m{L->ia, L->ja, L->a, nullptr, L->nnz};
        SPT_CUDA((launch_chunk<double, OUT_SET64>(m, n, b, x32, x, st, sms, stream)));
        long long rgrid = ((long long)n * 32 + 255) / 256;  // one warp per row, at most 16 blocks per SM
        if (rgrid > 16LL * sms) rgrid = 16LL * sms;
        for (int it = 0; it < ir_iters; it++) {
            k_residual_nat<<<(int)rgrid, 256, 0, stream>>>(L->ia, L->ja, L->a, n, L->nnz, b, x, r32, st);
            SPT_CUDA(cudaGetLastError());
            SPT_CUDA(cudaMemsetAsync(x32, 0xFF, sizeof(float) * (size_t)n, stream));
            SPT_CUDA((launch_chunk<float, OUT_ADD64>(m, n, r32, x32, x, st, sms, stream)));
        }
        DevStatus h{};
        SPT_CUDA(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, stream));
        SPT_CUDA(cudaStreamSynchronize(stream));
        if (h.code == SPTRSV_ERR_INVALID_CSR)
            return set_error(SPTRSV_ERR_INVALID_CSR,
                             "solve_ir_noalloc: row %d is not lower-triangular CSR with the diagonal last", h.row);
        if (h.code == SPTRSV_ERR_TIMEOUT)
            return set_error(SPTRSV_ERR_TIMEOUT, "solve_ir_noalloc: device wait ran out of budget at row %d", h.row);
        if (h.code != 0) return set_error(h.code, "solve_ir_noalloc: device error %d at row %d", h.code, h.row);
        return ok();
    });
}
