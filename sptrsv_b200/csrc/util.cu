// util.cu — device-wide exclusive scan and stable LSD radix sort (int keys).
//
// The analysis needs a stable sort of rows by key (the reference uses
// thrust::stable_sort_by_key, analysis/analysis_csr.cu:352) and exclusive
// scans of bucket counts (:370-374).  Both are written here from scratch:
//  - scan: three phases over tiles of 4096 ints (tile sums, one-block scan
//    of the tile sums, tile scan plus offset);
//  - radix sort: 4-bit digits, LSD.  Each pass builds a digit x tile count
//    table, scans it digit-major (so equal digits keep tile order) and
//    scatters; inside a tile every thread owns 16 consecutive items and
//    ranks them with packed 16-bit counters and a block scan, which keeps
//    equal digits in index order.  The whole sort is therefore stable.
#include "internal.h"

namespace sptrsv {

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one int per thread; returns the block total.
template <int NT>
__device__ __forceinline__ int block_exclusive_scan(int v, int* smem_warp, int& total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) smem_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int w = lane < NT / 32 ? smem_warp[lane] : 0;
        int winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= o) winc += t;
        }
        if (lane < NT / 32) smem_warp[lane] = winc - w;
        if (lane == NT / 32 - 1) smem_warp[32] = winc;
    }
    __syncthreads();
    int r = smem_warp[wid] + inc - v;
    total = smem_warp[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tile_sums(const int* __restrict__ in, long long m,
                                                                 int* __restrict__ sums)
{
    __shared__ int sw[33];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++)
        if (base + j < m) s += in[base + j];
    int total;
    block_exclusive_scan<kScanThreads>(s, sw, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block scans the tile sums in place (exclusive), 512 at a time.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int* sums, int nb)
{
    __shared__ int sw[33];
    int carry = 0;
    for (int base = 0; base < nb; base += kScanThreads) {
        int i = base + threadIdx.x;
        int v = i < nb ? sums[i] : 0;
        int total;
        int ex = block_exclusive_scan<kScanThreads>(v, sw, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int* in, int* out, long long m,
                                                             const int* __restrict__ offs)
{
    __shared__ int sw[33];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        v[j] = base + j < m ? in[base + j] : 0;
        s += v[j];
    }
    int total;
    int ex = block_exclusive_scan<kScanThreads>(s, sw, total) + offs[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        if (base + j < m) out[base + j] = ex;
        ex += v[j];
    }
}

constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;
constexpr int kRadixBins = 16;

__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const int* __restrict__ keys, long long n, int shift,
                                                              int* __restrict__ hist, int ntiles)
{
    __shared__ int h[kRadixBins];
    if (threadIdx.x < kRadixBins) h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kRadixTile + (long long)threadIdx.x * kRadixItems;
    int cnt[kRadixBins];
#pragma unroll
    for (int d = 0; d < kRadixBins; d++) cnt[d] = 0;
#pragma unroll
    for (int j = 0; j < kRadixItems; j++)
        if (base + j < n) {
            int d = (keys[base + j] >> shift) & (kRadixBins - 1);
#pragma unroll
            for (int q = 0; q < kRadixBins; q++) cnt[q] += (q == d);
        }
#pragma unroll
    for (int d = 0; d < kRadixBins; d++)
        if (cnt[d]) atomicAdd(&h[d], cnt[d]);
    __syncthreads();
    if (threadIdx.x < kRadixBins) hist[(long long)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Block exclusive scan of 8 packed words (16 digits x 16 bits) per thread.
__device__ __forceinline__ void block_scan_packed(unsigned (&w)[8], unsigned (*sw)[8])
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned inc[8];
#pragma unroll
    for (int q = 0; q < 8; q++) inc[q] = w[q];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int q = 0; q < 8; q++) {
            unsigned t = __shfl_up_sync(0xffffffffu, inc[q], o);
            if (lane >= o) inc[q] += t;
        }
    }
    if (lane == 31)
#pragma unroll
        for (int q = 0; q < 8; q++) sw[wid][q] = inc[q];
    __syncthreads();
    unsigned pre[8];
#pragma unroll
    for (int q = 0; q < 8; q++) pre[q] = 0;
    for (int k = 0; k < wid; k++)
#pragma unroll
        for (int q = 0; q < 8; q++) pre[q] += sw[k][q];
#pragma unroll
    for (int q = 0; q < 8; q++) w[q] = pre[q] + inc[q] - w[q];
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(const int* __restrict__ kin, const int* __restrict__ vin,
                                                                 int* __restrict__ kout, int* __restrict__ vout,
                                                                 long long n, int shift, const int* __restrict__ offs,
                                                                 int ntiles)
{
    __shared__ unsigned sw[kRadixThreads / 32][8];
    long long base = (long long)blockIdx.x * kRadixTile + (long long)threadIdx.x * kRadixItems;
    int key[kRadixItems], val[kRadixItems];
    unsigned char rank[kRadixItems];
    unsigned w[8];
#pragma unroll
    for (int q = 0; q < 8; q++) w[q] = 0;
#pragma unroll
    for (int j = 0; j < kRadixItems; j++) {
        bool in = base + j < n;
        key[j] = in ? kin[base + j] : 0;
        val[j] = in ? vin[base + j] : 0;
        int d = (key[j] >> shift) & (kRadixBins - 1);
        unsigned c = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            unsigned lo = w[q] & 0xFFFFu, hi = w[q] >> 16;
            if (2 * q == d) c = lo;
            if (2 * q + 1 == d) c = hi;
        }
        rank[j] = (unsigned char)c;
        if (in) {
#pragma unroll
            for (int q = 0; q < 8; q++) w[q] += (2 * q == d ? 1u : 0u) + (2 * q + 1 == d ? 0x10000u : 0u);
        }
    }
    block_scan_packed(w, sw);
#pragma unroll
    for (int j = 0; j < kRadixItems; j++) {
        if (base + j < n) {
            int d = (key[j] >> shift) & (kRadixBins - 1);
            unsigned ex = 0;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (2 * q == d) ex = w[q] & 0xFFFFu;
                if (2 * q + 1 == d) ex = w[q] >> 16;
            }
            long long pos = (long long)offs[(long long)d * ntiles + blockIdx.x] + ex + rank[j];
            kout[pos] = key[j];
            vout[pos] = val[j];
        }
    }
}

__global__ void k_seg_count(const int* __restrict__ key, int n, int* __restrict__ cnt)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int k = key[p];
        unsigned peers = __match_any_sync(__activemask(), k);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(cnt + k, __popc(peers));
    }
}

// rows per task of a segment: R, or 32 >> (key % 6) when R <= 0
__device__ __forceinline__ int task_rows(int R, int key) { return R > 0 ? R : (32 >> (key % 6)); }

__global__ void k_task_flags(const int* __restrict__ key, const int* __restrict__ seg_ptr, int n, int R,
                             int* __restrict__ flag)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= n; p += gridDim.x * blockDim.x)
        flag[p] = p < n ? ((p - seg_ptr[key[p]]) % task_rows(R, key[p]) == 0) : 0;
}

__global__ void k_task_base(const int* __restrict__ flag_scan, const int* __restrict__ key,
                            const int* __restrict__ seg_ptr, int n, int R, int* __restrict__ tbase)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= n; p += gridDim.x * blockDim.x) {
        if (p == n) tbase[flag_scan[n]] = n;
        else if ((p - seg_ptr[key[p]]) % task_rows(R, key[p]) == 0) tbase[flag_scan[p]] = p;
    }
}

}  // namespace

int build_task_table(const int* key, int n, int K, int R, int** tbase, int* ntasks, cudaStream_t s)
{
    *tbase = nullptr;
    *ntasks = 0;
    int *cnt = nullptr, *flag = nullptr, *scr = nullptr;
    auto cleanup = [&]() {
        cudaFree(cnt);
        cudaFree(flag);
        cudaFree(scr);
    };
#define TCHK(call)                                   \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) {                     \
            cleanup();                               \
            return cuda_fail(e_, #call);             \
        }                                            \
    } while (0)
    long long sn = scan_scratch_ints((long long)(n > K ? n : K) + 1);
    TCHK(dalloc(&cnt, (long long)K + 1));
    TCHK(dalloc(&flag, (long long)n + 1));
    TCHK(dalloc(&scr, sn));
    TCHK(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)K + 1), s));
    if (n > 0) {
        k_seg_count<<<grid_for(n, 256), 256, 0, s>>>(key, n, cnt);
        TCHK(cudaGetLastError());
    }
    TCHK(scan_exclusive(cnt, cnt, (long long)K + 1, scr, s));  // cnt -> segment starts
    k_task_flags<<<grid_for((long long)n + 1, 256), 256, 0, s>>>(key, cnt, n, R, flag);
    TCHK(cudaGetLastError());
    TCHK(scan_exclusive(flag, flag, (long long)n + 1, scr, s));
    int nt = 0;
    TCHK(cudaMemcpyAsync(&nt, flag + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    TCHK(cudaStreamSynchronize(s));
    TCHK(dalloc(tbase, (long long)nt + 1));
    k_task_base<<<grid_for((long long)n + 1, 256), 256, 0, s>>>(flag, key, cnt, n, R, *tbase);
    TCHK(cudaGetLastError());
    TCHK(cudaStreamSynchronize(s));
#undef TCHK
    cleanup();
    *ntasks = nt;
    return 0;
}

long long scan_scratch_ints(long long m) { return (m + kScanTile - 1) / kScanTile + 1; }

cudaError_t scan_exclusive(const int* in, int* out, long long m, int* scratch, cudaStream_t s)
{
    if (m <= 0) return cudaSuccess;
    int nb = (int)((m + kScanTile - 1) / kScanTile);
    k_scan_tile_sums<<<nb, kScanThreads, 0, s>>>(in, m, scratch);
    k_scan_sums<<<1, kScanThreads, 0, s>>>(scratch, nb);
    k_scan_apply<<<nb, kScanThreads, 0, s>>>(in, out, m, scratch);
    return cudaGetLastError();
}

long long radix_scratch_ints(long long n)
{
    long long nt = (n + kRadixTile - 1) / kRadixTile;
    long long h = nt * kRadixBins;
    return h + scan_scratch_ints(h);
}

cudaError_t radix_sort_pairs(int* keys, int* vals, int* keys_tmp, int* vals_tmp, long long n, int max_key,
                             int* scratch, cudaStream_t s)
{
    if (n <= 1 || max_key <= 0) return cudaSuccess;
    int bits = 32 - __builtin_clz((unsigned)max_key);
    int passes = (bits + 3) / 4;
    int ntiles = (int)((n + kRadixTile - 1) / kRadixTile);
    long long h = (long long)ntiles * kRadixBins;
    int* hist = scratch;
    int* sscr = scratch + h;
    int *ka = keys, *va = vals, *kb = keys_tmp, *vb = vals_tmp;
    for (int p = 0; p < passes; p++) {
        int shift = 4 * p;
        k_radix_hist<<<ntiles, kRadixThreads, 0, s>>>(ka, n, shift, hist, ntiles);
        cudaError_t e = scan_exclusive(hist, hist, h, sscr, s);
        if (e != cudaSuccess) return e;
        k_radix_scatter<<<ntiles, kRadixThreads, 0, s>>>(ka, va, kb, vb, n, shift, hist, ntiles);
        int* t = ka; ka = kb; kb = t;
        t = va; va = vb; vb = t;
    }
    if (ka != keys) {
        cudaMemcpyAsync(keys, ka, sizeof(int) * n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(vals, va, sizeof(int) * n, cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

}  // namespace sptrsv
