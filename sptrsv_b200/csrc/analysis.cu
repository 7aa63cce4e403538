// analysis.cu — GPU analysis pass, bit-exact with the reference's
// multirow_analysis_base_GPU (analysis/analysis_csr.cu:272-410).
//
// Steps (reference line in brackets):
//  0. CSR validation: lower triangular, sorted columns, diagonal last.  The
//     reference trusts its input and hangs on a bad one; here a bad matrix
//     is an error return.
//  1. Levels [:104-185]: level[i] = 1 + max(level[j]) over the off-diagonal
//     columns j of row i.  This is a max-plus triangular solve, done with the
//     same sync-free pattern as the numeric solve: a persistent grid walks the
//     rows in natural order (a topological order), each row polls its
//     dependencies' levels (0 = not yet written) with bounded relaxed loads.
//     nlevs = max level [:305] via one atomicMax per warp.
//  2. Key = 7*(level-1) + bucket(offdiag count) [:12-32, :53-57, :307-332]
//     and per-key row counts (the reference's sort + reduce_by_key + scatter,
//     :336-348) with warp-aggregated atomics.
//  3. iorder = rows stably sorted by key [:350-352]: the stable LSD radix
//     sort of util.cu on (key, row).
//  4. Multirow warp map [:354-385, kernel_base :244-270]: warps per key =
//     ceil(count * lanes / 32), two exclusive scans, then one thread per warp
//     writes ibase_row / ivect_size_warp.
#include <cstdlib>
#include <cstring>

#include "internal.h"

namespace sptrsv {

namespace {

// bucket of a row by its off-diagonal count (vect_size_calculator, :12-32)
__device__ __forceinline__ int bucket_of(int nnz_off)
{
    if (nnz_off == 0) return 6;
    if (nnz_off == 1) return 0;
    if (nnz_off <= 2) return 1;
    if (nnz_off <= 4) return 2;
    if (nnz_off <= 8) return 3;
    if (nnz_off <= 16) return 4;
    return 5;
}

// res[0] = error flag, res[1] = first bad row (starts at INT_MAX)
__global__ void k_validate(const int* __restrict__ rowptr, const int* __restrict__ col, int n, int nnz, int* res)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int s = rowptr[i], e = rowptr[i + 1];
        bool bad = (i == 0 && s != 0) || e <= s || e > nnz || s < 0;
        if (!bad) {
            bad = col[e - 1] != i;
            int prev = -1;
            for (int p = s; p < e - 1 && !bad; p++) {
                int c = col[p];
                if (c <= prev || c >= i) bad = true;
                prev = c;
            }
        }
        if (bad) {
            atomicOr(res, 1);
            atomicMin(res + 1, i);
        }
    }
}

// Persistent sync-free level computation over natural-order chunks: warp
// task t covers rows [32t, 32t+32) and computes them one after another, all
// 32 lanes striding a row's columns.  Natural order is topological, so a
// dependency inside the chunk was computed by this warp a moment ago and is
// read from the warp's shared-memory ring; a dependency outside is polled
// warp-convergently (level 0 = not yet written).  Row metadata of the whole
// chunk is loaded up front, one row per lane.
// With a task table (task_r0 != null), task t covers rows [task_r0[t],
// task_r0[t] + task_cnt[t]) instead (at most 32 consecutive rows); any
// order in which every row's dependencies lie in earlier tasks or earlier in
// its own task is deadlock-free.
__global__ void __launch_bounds__(256) k_levels(const int* __restrict__ rowptr, const int* __restrict__ col, int n,
                                                int* level, int* nlevs, DevStatus* st, unsigned long long budget,
                                                const int* __restrict__ task_r0, const int* __restrict__ task_cnt,
                                                long long ntask)
{
    __shared__ int ring[8][32];
    const int lane = threadIdx.x & 31;
    int* my = ring[threadIdx.x >> 5];
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long ntasks = task_r0 ? ntask : ((long long)n + 31) / 32;
    int my_max = 0;
    for (long long t = gw; t < ntasks; t += nw) {
        const int r0 = task_r0 ? __ldg(task_r0 + t) : (int)(t * 32);
        const int cnt = task_r0 ? __ldg(task_cnt + t) : min(32, n - r0);
        int ms = 0, me = 0;
        if (lane < cnt) {
            ms = __ldg(rowptr + r0 + lane);
            me = __ldg(rowptr + r0 + lane + 1) - 1;
        }
        for (int j = 0; j < cnt; j++) {
            const int s = __shfl_sync(0xffffffffu, ms, j), e = __shfl_sync(0xffffffffu, me, j);
            int m = 0;
            for (int p = s + lane; __any_sync(0xffffffffu, p < e); p += 32) {
                const bool have = p < e;
                const int c = have ? __ldg(col + p) : 0;
                const bool local = have && c >= r0;
                int lv = local ? my[c - r0] : 0;
                if (!warp_wait<false, int>(have && !local, c, level, nullptr, lv, st, budget, 0u, r0 + j)) return;
                if (have) m = max(m, lv);
            }
            m = __reduce_max_sync(0xffffffffu, m);
            if (lane == 0) {
                my[j] = m + 1;
                st_relaxed(level + r0 + j, m + 1);
            }
            my_max = max(my_max, m + 1);
            __syncwarp();
        }
    }
    if (lane == 0 && my_max > 0) atomicMax(nlevs, my_max);
}

__global__ void k_keys(const int* __restrict__ rowptr, const int* __restrict__ level, int n, int* __restrict__ key,
                       int* __restrict__ iota, int* counts)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int k = 7 * (level[i] - 1) + bucket_of(rowptr[i + 1] - rowptr[i] - 1);
        key[i] = k;
        iota[i] = i;
        unsigned peers = __match_any_sync(__activemask(), k);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(counts + k, __popc(peers));
    }
}

// warps per key (get_warps_per_bucks :66-71 with get_size_from_pos :84-102)
__global__ void k_warps_per_key(const int* __restrict__ counts, int K, int* __restrict__ wpk)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= K; k += gridDim.x * blockDim.x) {
        if (k == K) {
            wpk[k] = 0;
            continue;
        }
        int b = k % 7;
        int sz = b == 6 ? 1 : (1 << b);
        wpk[k] = (int)(((long long)counts[k] * sz + 31) / 32);
    }
}

// one thread per multirow warp (kernel_base :244-270)
__global__ void k_warp_map(const int* __restrict__ warp_off, const int* __restrict__ row_off, int K, int n_warps,
                           int n, int* __restrict__ ibase, int* __restrict__ ivect, int* __restrict__ wlev)
{
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n_warps; w += gridDim.x * blockDim.x) {
        int lo = 0, hi = K - 1;  // largest k with warp_off[k] <= w
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (warp_off[mid] <= w) lo = mid;
            else hi = mid - 1;
        }
        int k = lo, b = k % 7;
        int size = b == 6 ? 0 : (1 << b);
        int sz = size == 0 ? 1 : size;
        ibase[w] = row_off[k] + (w - warp_off[k]) * (32 / sz);
        ivect[w] = size;
        wlev[w] = k / 7 + 1;
        if (w == 0) ibase[n_warps] = n;
    }
}

__global__ void k_level_sizes(const int* __restrict__ counts, int nlevs, int* __restrict__ lev_size)
{
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nlevs; l += gridDim.x * blockDim.x) {
        int s = 0;
        for (int b = 0; b < 7; b++) s += counts[7 * l + b];
        lev_size[l] = s;
    }
}

__global__ void k_inverse(const int* __restrict__ perm, int n, int* __restrict__ inv)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) inv[perm[k]] = k;
}



}  // namespace

// Checks a device CSR; returns 0, SPTRSV_ERR_INVALID_CSR (with *bad_row) or a CUDA error code.
int validate_csr_device(const int* rowptr, const int* col, int n, int nnz, cudaStream_t s, int* bad_row)
{
    *bad_row = -1;
    if (n <= 0) return 0;
    int* d_res = nullptr;
    SPT_CUDA(cudaMalloc((void**)&d_res, 2 * sizeof(int)));
    int h[2] = {0, 0x7fffffff};
    cudaError_t e = cudaMemcpyAsync(d_res, h, sizeof(h), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_validate<<<grid_for(n, 256), 256, 0, s>>>(rowptr, col, n, nnz, d_res);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_res, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_res);
    if (e != cudaSuccess) return cuda_fail(e, "validate_csr_device");
    if (h[0]) {
        *bad_row = h[1];
        return SPTRSV_ERR_INVALID_CSR;
    }
    return 0;
}

// Runs the whole analysis; fills *info per `mode` and registers the record.
int run_analysis_impl(dfr_analysis_info_t* info, const sp_mat_t* L, MODE mode, const LevelTasks* tasks)
{
    if (!info || !L) return set_error(SPTRSV_ERR_INVALID_ARG, "analysis: NULL info or matrix");
    const int n = L->nr;
    if (n < 0 || L->nc != n || L->nnz < n) return set_error(SPTRSV_ERR_INVALID_ARG, "analysis: bad sizes n=%d nnz=%d", n, L->nnz);
    if (n > 0 && (!L->ia || !L->ja)) return set_error(SPTRSV_ERR_INVALID_ARG, "analysis: NULL device arrays");
    Ctx* c = ctx();
    if (!c) return set_error(SPTRSV_ERR_CUDA, "analysis: no CUDA device");
    cudaStream_t s = 0;
    const int nnz = L->nnz;

    // 0. validation (the status block must be clean before the bounded waits)
    {
        int e = sync_status(s);
        if (e) return e;
        int bad = -1;
        e = validate_csr_device(L->ia, L->ja, n, nnz, s, &bad);
        if (e == SPTRSV_ERR_INVALID_CSR)
            return set_error(e, "analysis: row %d is not lower-triangular CSR with sorted columns and the diagonal last",
                             bad);
        if (e) return e;
    }

    AnalysisRec* rec = new AnalysisRec();
    rec->device = c->device;
    rec->n = n;
    rec->nnz = nnz;
    int *d_key = nullptr, *d_key2 = nullptr, *d_val2 = nullptr, *d_scr = nullptr, *d_nlevs = nullptr;
    int *d_iorder = nullptr, *d_rowctr = nullptr, *d_levsz = nullptr, *d_inv = nullptr;
    int *d_wpk = nullptr, *d_rowoff = nullptr;
    auto fail = [&](int code) {
        cudaFree(d_key); cudaFree(d_key2); cudaFree(d_val2); cudaFree(d_scr); cudaFree(d_nlevs);
        cudaFree(d_iorder); cudaFree(d_rowctr); cudaFree(d_levsz); cudaFree(d_inv);
        cudaFree(d_wpk); cudaFree(d_rowoff);
        cudaFree(rec->d_levels); cudaFree(rec->d_counts); cudaFree(rec->d_ibase); cudaFree(rec->d_ivect);
        cudaFree(rec->d_wlev);
        delete rec;
        return code;
    };
#define ACHK(call)                                              \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, #call)); \
    } while (0)

    ACHK(dalloc(&rec->d_levels, n));
    ACHK(dalloc(&d_nlevs, 1));
    ACHK(dalloc(&d_iorder, n));
    ACHK(dalloc(&d_rowctr, 1));
    ACHK(cudaMemsetAsync(rec->d_levels, 0, sizeof(int) * (size_t)(n > 0 ? n : 1), s));
    ACHK(cudaMemsetAsync(d_nlevs, 0, sizeof(int), s));
    ACHK(cudaMemsetAsync(d_rowctr, 0, sizeof(int), s));

    // 1. levels
    int nlevs = 0;
    if (n > 0) {
        // one 32-row chunk per warp, 8 warps per block
        const long long nt = tasks ? tasks->n : ((long long)n + 31) / 32;
        ACHK(launch_persistent(k_levels, 256, 0, (nt + 7) / 8, s, L->ia, L->ja, n, rec->d_levels, d_nlevs,
                               c->d_status, wait_budget_ns(), tasks ? tasks->r0 : (const int*)nullptr,
                               tasks ? tasks->cnt : (const int*)nullptr, nt));
        ACHK(cudaMemcpyAsync(&nlevs, d_nlevs, sizeof(int), cudaMemcpyDeviceToHost, s));
        int st = sync_status(s);
        if (st) return fail(st);
    }
    rec->nlevs = nlevs;
    const long long K = 7LL * nlevs;

    // 2-3. keys, counts, stable sort
    ACHK(dalloc(&rec->d_counts, K + 1));
    ACHK(cudaMemsetAsync(rec->d_counts, 0, sizeof(int) * (size_t)(K + 1), s));
    ACHK(dalloc(&d_key, n));
    ACHK(dalloc(&d_key2, n));
    ACHK(dalloc(&d_val2, n));
    long long scr = radix_scratch_ints(n);
    long long scr2 = scan_scratch_ints(K + 1);
    ACHK(dalloc(&d_scr, scr > scr2 ? scr : scr2));
    if (n > 0) {
        k_keys<<<grid_for(n, 256), 256, 0, s>>>(L->ia, rec->d_levels, n, d_key, d_iorder, rec->d_counts);
        ACHK(cudaGetLastError());
        ACHK(radix_sort_pairs(d_key, d_iorder, d_key2, d_val2, n, (int)(K - 1), d_scr, s));
    }

    // 4. multirow warp map (always built; exposed in info for MULTIROW/ALL)
    ACHK(dalloc(&d_wpk, K + 1));
    ACHK(dalloc(&d_rowoff, K + 1));
    int n_warps = 0;
    if (K > 0) {
        k_warps_per_key<<<grid_for(K + 1, 256), 256, 0, s>>>(rec->d_counts, (int)K, d_wpk);
        ACHK(cudaGetLastError());
        ACHK(scan_exclusive(d_wpk, d_wpk, K + 1, d_scr, s));
        ACHK(scan_exclusive(rec->d_counts, d_rowoff, K + 1, d_scr, s));
        ACHK(cudaMemcpyAsync(&n_warps, d_wpk + K, sizeof(int), cudaMemcpyDeviceToHost, s));
        ACHK(cudaStreamSynchronize(s));
    }
    rec->n_warps = n_warps;
    ACHK(dalloc(&rec->d_ibase, (long long)n_warps + 1));
    ACHK(dalloc(&rec->d_ivect, n_warps));
    ACHK(dalloc(&rec->d_wlev, n_warps));
    if (n_warps > 0) {
        k_warp_map<<<grid_for(n_warps, 256), 256, 0, s>>>(d_wpk, d_rowoff, (int)K, n_warps, n, rec->d_ibase,
                                                           rec->d_ivect, rec->d_wlev);
        ACHK(cudaGetLastError());
    } else {
        ACHK(cudaMemsetAsync(rec->d_ibase, 0, sizeof(int), s));
    }

    // extras the reference declares but never fills
    ACHK(dalloc(&d_levsz, nlevs));
    ACHK(dalloc(&d_inv, n));
    if (nlevs > 0) {
        k_level_sizes<<<grid_for(nlevs, 256), 256, 0, s>>>(rec->d_counts, nlevs, d_levsz);
        ACHK(cudaGetLastError());
    }
    if (n > 0) {
        k_inverse<<<grid_for(n, 256), 256, 0, s>>>(d_iorder, n, d_inv);
        ACHK(cudaGetLastError());
    }
    ACHK(cudaStreamSynchronize(s));
    cudaFree(d_key);
    cudaFree(d_key2);
    cudaFree(d_val2);
    cudaFree(d_scr);
    cudaFree(d_nlevs);
    cudaFree(d_wpk);
    cudaFree(d_rowoff);
#undef ACHK

    info->mode = mode;
    info->lev_ctr = 0;
    info->nlevs = nlevs;
    info->lev_size = d_levsz;
    info->inv_iorder = d_inv;
    info->iorder = d_iorder;
    info->row_ctr = d_rowctr;
    if (mode == MULTIROW || mode == ALL) {
        info->n_warps = n_warps;
        info->ibase_row = rec->d_ibase;
        info->ivect_size_warp = rec->d_ivect;
        info->warp_lev = rec->d_wlev;
        rec->map_in_info = true;
    } else {
        info->n_warps = 0;
        info->ibase_row = nullptr;
        info->ivect_size_warp = nullptr;
        info->warp_lev = nullptr;
        rec->map_in_info = false;
    }
    register_analysis(d_rowctr, rec);
    return ok();
}

}  // namespace sptrsv
