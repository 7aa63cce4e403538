// features.cu — the 12 cheap analysis features the schedule selector reads.
//
//   0 log2 n                 6  q25 of off-diagonals per row
//   1 log2 nnz               7  q50
//   2 nnz / n                8  q90
//   3 log2 nlevs             9  q99
//   4 log2 (n / nlevs)      10  log2 (1 + max off-diagonals per row)
//   5 log2 max level width  11  fraction of diagonal-only rows
//
// Row lengths go into a histogram with exact bins below 256 and one bin per
// power of two above; quantiles read the histogram (exact below 256, the bin's
// lower edge above).  Level widths come from the analysis' per-level sizes.
#include <cmath>
#include <vector>

#include "internal.h"

namespace sptrsv {

namespace {

constexpr int kExact = 256;
constexpr int kBins = kExact + 24;

__device__ __forceinline__ int len_bin(int l)
{
    if (l < kExact) return l;
    int lg = 31 - __clz(l);  // >= 8
    return min(kExact + lg - 8, kBins - 1);
}

__global__ void k_len_hist(const int* __restrict__ rowptr, int n, int* __restrict__ hist, int* __restrict__ maxlen)
{
    __shared__ int h[kBins];
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    int mx = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int l = rowptr[i + 1] - rowptr[i] - 1;
        atomicAdd(&h[len_bin(l)], 1);
        mx = max(mx, l);
    }
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxlen, mx);
    __syncthreads();
    for (int i = threadIdx.x; i < kBins; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void k_max(const int* __restrict__ a, int m, int* __restrict__ out)
{
    int mx = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) mx = max(mx, a[i]);
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

double quantile(const std::vector<int>& h, long long n, double q)
{
    long long target = (long long)std::ceil(q * (double)n);
    if (target < 1) target = 1;
    long long acc = 0;
    for (int b = 0; b < kBins; b++) {
        acc += h[b];
        if (acc >= target) return b < kExact ? (double)b : std::ldexp(1.0, b - kExact + 8);
    }
    return 0.0;
}

}  // namespace

int compute_features(const sp_mat_t* L, const dfr_analysis_info_t* info, float* out)
{
    const int n = L->nr;
    if (n <= 0) return set_error(SPTRSV_ERR_INVALID_ARG, "features: empty matrix");
    int* d = nullptr;  // [kBins] hist, [1] max len, [1] max level width
    SPT_CUDA(cudaMalloc((void**)&d, sizeof(int) * (kBins + 2)));
    cudaError_t e = cudaMemset(d, 0, sizeof(int) * (kBins + 2));
    if (e == cudaSuccess) {
        k_len_hist<<<grid_for(n, 256), 256>>>(L->ia, n, d, d + kBins);
        if (info->lev_size && info->nlevs > 0) k_max<<<grid_for(info->nlevs, 256), 256>>>(info->lev_size, info->nlevs, d + kBins + 1);
        e = cudaGetLastError();
    }
    std::vector<int> h(kBins + 2, 0);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, sizeof(int) * (kBins + 2), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "features");
    const double nn = (double)n, nnz = (double)L->nnz, nl = (double)(info->nlevs > 0 ? info->nlevs : 1);
    out[0] = (float)std::log2(nn);
    out[1] = (float)std::log2(nnz);
    out[2] = (float)(nnz / nn);
    out[3] = (float)std::log2(nl);
    out[4] = (float)std::log2(nn / nl);
    out[5] = (float)std::log2((double)(h[kBins + 1] > 0 ? h[kBins + 1] : 1));
    out[6] = (float)quantile(h, n, 0.25);
    out[7] = (float)quantile(h, n, 0.50);
    out[8] = (float)quantile(h, n, 0.90);
    out[9] = (float)quantile(h, n, 0.99);
    out[10] = (float)std::log2(1.0 + (double)h[kBins]);
    out[11] = (float)((double)h[0] / nn);
    return 0;
}

}  // namespace sptrsv

extern "C" int sptrsv_features(const sp_mat_t* L, const dfr_analysis_info_t* info, float* out12)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!L || !info || !out12) return sptrsv::set_error(SPTRSV_ERR_INVALID_ARG, "features: NULL argument");
        if (!info->iorder) return sptrsv::set_error(SPTRSV_ERR_NOT_ANALYSED, "features: info is not analysed");
        int e = sptrsv::compute_features(L, info, out12);
        return e ? e : sptrsv::ok();
    });
}
