// cluster.cu — the cluster layout of a plan.
//
// Deep, narrow dependency graphs (a 2D grid has one level per anti-diagonal)
// spend their time on the chain of dependent rows, and each link of that
// chain costs an L2 round trip when producer and consumer sit on different
// SMs.  The cluster schedule makes most links shared-memory hops:
//   1. band(i) = (level(i)-1) / H cuts the level order into bands of H levels;
//   2. inside a band, rows are taken in natural-index order and cut into
//      clusters of at most B rows;
//   3. the layout order is (cluster, level, natural index).
// Any contiguous range of the (band, natural index) order is a topological
// order of a lower-triangular matrix, so every cross-cluster dependency
// points to an earlier cluster and clusters can be processed in order by
// persistent CTAs without deadlock.  Natural-index locality (banded and
// grid matrices couple nearby rows) makes a cluster a compact region of the
// graph: for the 2048x2048 grid with H = 64, B = 4096 a cluster is a 64x64
// parallelogram and a longest path crosses ~128 cluster boundaries instead
// of 4095 SM boundaries.
//
// Columns of the cluster layout are encoded: c >= 0 is an original row (its
// value is read from x in global memory), c < 0 names local position ~c of
// the same cluster (its value is in the CTA's shared memory).
#include "internal.h"
#include "plan.h"

namespace sptrsv {

namespace {

__global__ void k_band_keys(const int* __restrict__ level, int n, int H, int* __restrict__ key, int* __restrict__ iota,
                            int* __restrict__ band_cnt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = (level[i] - 1) / H;
        key[i] = b;
        iota[i] = i;
        unsigned peers = __match_any_sync(__activemask(), b);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(band_cnt + b, __popc(peers));
    }
}

__global__ void k_clusters_per_band(const int* __restrict__ band_cnt, int nb, int B, int* __restrict__ cpb)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nb; b += gridDim.x * blockDim.x)
        cpb[b] = b < nb ? (band_cnt[b] + B - 1) / B : 0;
}

// position p of the (band, natural) order -> cluster id and final sort key
__global__ void k_assign_clusters(const int* __restrict__ s1, const int* __restrict__ key_sorted,
                                  const int* __restrict__ band_start, const int* __restrict__ band_coff,
                                  const int* __restrict__ level, int n, int H, int B, int* __restrict__ cl,
                                  int* __restrict__ key2, int* __restrict__ ccnt)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int r = s1[p];
        int b = key_sorted[p];
        int cid = band_coff[b] + (p - band_start[b]) / B;
        cl[r] = cid;
        key2[r] = cid * H + (level[r] - 1 - b * H);
        unsigned peers = __match_any_sync(__activemask(), cid);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(ccnt + cid, __popc(peers));
    }
}

__global__ void k_iota(int* a, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

__global__ void k_cluster_rows(const int* __restrict__ order, const int* __restrict__ lev_inv,
                               const int* __restrict__ lev_ptr, int n, int* __restrict__ len, int* __restrict__ rowid,
                               int* __restrict__ pos_of)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x) {
        if (k == n) {
            len[k] = 0;
            continue;
        }
        int r = order[k];
        int q = lev_inv[r];
        rowid[k] = r;
        pos_of[r] = k;
        len[k] = lev_ptr[q + 1] - lev_ptr[q];
    }
}

// one warp per cluster-layout position: copy the row from the level layout,
// encoding columns that fall in the same cluster as local positions
__global__ void k_cluster_fill(SptLayout lev, const int* __restrict__ lev_inv, SptLayout clu,
                               const int* __restrict__ cl, const int* __restrict__ pos_of,
                               const int* __restrict__ cptr, int n)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long k = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nw) {
        int r = clu.rowid[k];
        int q = lev_inv[r];
        int s = lev.ptr[q], e = lev.ptr[q + 1], o = clu.ptr[k];
        int my = cl[r];
        int base = cptr[my];
        for (int p = s + lane; p < e; p += 32) {
            int c = lev.col[p];
            int enc = cl[c] == my ? ~(pos_of[c] - base) : c;
            clu.col[o + p - s] = enc;
            clu.val64[o + p - s] = lev.val64[p];
            clu.val32[o + p - s] = lev.val32[p];
        }
        if (lane == 0) {
            clu.dg64[k] = lev.dg64[q];
            clu.dg32[k] = lev.dg32[q];
            clu.di64[k] = lev.di64[q];
            clu.di32[k] = lev.di32[q];
        }
    }
}

__global__ void k_level_keys(const int* __restrict__ rowid, const int* __restrict__ level, int n, int* __restrict__ key)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) key[p] = level[rowid[p]] - 1;
}

// ctask[c] = first task whose base is >= cptr[c] (cluster starts are task starts)
__global__ void k_cluster_first_task(const int* __restrict__ cptr, int nclusters, const int* __restrict__ tbase,
                                     int ntasks, int* __restrict__ ctask)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= nclusters; c += gridDim.x * blockDim.x) {
        int v = cptr[c], lo = 0, hi = ntasks;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (tbase[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        ctask[c] = lo;
    }
}

}  // namespace

int build_order_tasks(sptrsv_plan_s* p, int R)
{
    int j = 0;
    while ((1 << j) < R) j++;
    if (p->ord_tasks[j]) return 0;
    int* key = nullptr;
    SPT_CUDA(dalloc(&key, p->n));
    if (p->n > 0) {
        k_level_keys<<<grid_for(p->n, 256), 256>>>(p->lev.rowid, p->levels, p->n, key);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            cudaFree(key);
            return cuda_fail(e, "order tasks");
        }
    }
    int rc = build_task_table(key, p->n, p->nlevs > 0 ? p->nlevs : 1, R, &p->ord_tasks[j], &p->ord_ntasks[j], 0);
    cudaFree(key);
    return rc;
}

int build_cluster_tasks(sptrsv_plan_s* p, int R)
{
    if (p->clu_tasks && p->clu_R == R) return 0;
    cudaFree(p->clu_tasks);
    cudaFree(p->clu_ctask);
    p->clu_tasks = p->clu_ctask = nullptr;
    p->clu_ntasks = 0;
    long long K = (long long)p->nclusters * p->clu_H;
    int rc = build_task_table(p->clu_key, p->n, (int)(K > 0 ? K : 1), R, &p->clu_tasks, &p->clu_ntasks, 0);
    if (rc) return rc;
    SPT_CUDA(dalloc(&p->clu_ctask, (long long)p->nclusters + 1));
    k_cluster_first_task<<<grid_for((long long)p->nclusters + 1, 256), 256>>>(p->cptr, p->nclusters, p->clu_tasks,
                                                                                p->clu_ntasks, p->clu_ctask);
    SPT_CUDA(cudaGetLastError());
    SPT_CUDA(cudaStreamSynchronize(0));
    p->clu_R = R;
    return 0;
}

void layout_free(SptLayout& l)
{
    cudaFree(l.ptr);
    cudaFree(l.rowid);
    cudaFree(l.col);
    cudaFree(l.val64);
    cudaFree(l.val32);
    cudaFree(l.dg64);
    cudaFree(l.dg32);
    cudaFree(l.di64);
    cudaFree(l.di32);
    l = SptLayout();
}

int layout_alloc(SptLayout& l, int n, int m)
{
    SPT_CUDA(dalloc(&l.ptr, (long long)n + 1));
    SPT_CUDA(dalloc(&l.rowid, n));
    SPT_CUDA(dalloc(&l.col, m));
    SPT_CUDA(dalloc(&l.val64, m));
    SPT_CUDA(dalloc(&l.val32, m));
    SPT_CUDA(dalloc(&l.dg64, n));
    SPT_CUDA(dalloc(&l.dg32, n));
    SPT_CUDA(dalloc(&l.di64, n));
    SPT_CUDA(dalloc(&l.di32, n));
    return 0;
}

int build_cluster_layout(sptrsv_plan_s* p, int H, int B)
{
    if (p->clu.ptr && p->clu_H == H && p->clu_B == B) return 0;
    layout_free(p->clu);
    cudaFree(p->cptr);
    cudaFree(p->clu_key);
    cudaFree(p->clu_tasks);
    cudaFree(p->clu_ctask);
    p->cptr = p->clu_key = p->clu_tasks = p->clu_ctask = nullptr;
    p->nclusters = p->clu_ntasks = p->clu_R = 0;
    const int n = p->n;
    if (n == 0) {
        p->clu_H = H;
        p->clu_B = B;
        return layout_alloc(p->clu, 0, 0);
    }
    cudaStream_t s = 0;
    const int nb = (p->nlevs + H - 1) / H;
    int *key = nullptr, *s1 = nullptr, *kt = nullptr, *vt = nullptr, *scr = nullptr, *band_cnt = nullptr;
    int *band_start = nullptr, *band_coff = nullptr, *cl = nullptr, *key2 = nullptr, *ord = nullptr;
    int *ccnt = nullptr, *pos_of = nullptr;
    int rc = 0;
    auto cleanup = [&]() {
        cudaFree(key); cudaFree(s1); cudaFree(kt); cudaFree(vt); cudaFree(scr); cudaFree(band_cnt);
        cudaFree(band_start); cudaFree(band_coff); cudaFree(cl); cudaFree(key2); cudaFree(ord);
        cudaFree(ccnt); cudaFree(pos_of);
    };
#define CCHK(call)                                  \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) {                    \
            rc = cuda_fail(e_, #call);              \
            cleanup();                              \
            return rc;                              \
        }                                           \
    } while (0)
    CCHK(dalloc(&key, n));
    CCHK(dalloc(&s1, n));
    CCHK(dalloc(&kt, n));
    CCHK(dalloc(&vt, n));
    long long scr_n = radix_scratch_ints(n);
    long long scr_b = scan_scratch_ints((long long)n + 1);
    CCHK(dalloc(&scr, scr_n > scr_b ? scr_n : scr_b));
    CCHK(dalloc(&band_cnt, (long long)nb + 1));
    CCHK(dalloc(&band_start, (long long)nb + 1));
    CCHK(dalloc(&band_coff, (long long)nb + 1));
    CCHK(cudaMemsetAsync(band_cnt, 0, sizeof(int) * ((size_t)nb + 1), s));
    // 1. rows in (band, natural) order
    k_band_keys<<<grid_for(n, 256), 256, 0, s>>>(p->levels, n, H, key, s1, band_cnt);
    CCHK(cudaGetLastError());
    CCHK(radix_sort_pairs(key, s1, kt, vt, n, nb - 1, scr, s));
    // 2. clusters per band
    CCHK(scan_exclusive(band_cnt, band_start, (long long)nb + 1, scr, s));
    k_clusters_per_band<<<grid_for((long long)nb + 1, 256), 256, 0, s>>>(band_cnt, nb, B, band_coff);
    CCHK(cudaGetLastError());
    CCHK(scan_exclusive(band_coff, band_coff, (long long)nb + 1, scr, s));
    int nclusters = 0;
    CCHK(cudaMemcpyAsync(&nclusters, band_coff + nb, sizeof(int), cudaMemcpyDeviceToHost, s));
    CCHK(cudaStreamSynchronize(s));
    // 3. cluster ids, final order (cluster, level, natural)
    CCHK(dalloc(&cl, n));
    CCHK(dalloc(&key2, n));
    CCHK(dalloc(&ord, n));
    CCHK(dalloc(&ccnt, (long long)nclusters + 1));
    CCHK(cudaMemsetAsync(ccnt, 0, sizeof(int) * ((size_t)nclusters + 1), s));
    k_assign_clusters<<<grid_for(n, 256), 256, 0, s>>>(s1, key, band_start, band_coff, p->levels, n, H, B, cl, key2,
                                                        ccnt);
    CCHK(cudaGetLastError());
    k_iota<<<grid_for(n, 256), 256, 0, s>>>(ord, n);
    CCHK(cudaGetLastError());
    long long maxkey = (long long)nclusters * H - 1;
    CCHK(radix_sort_pairs(key2, ord, kt, vt, n, (int)maxkey, scr, s));
    CCHK(dalloc(&p->cptr, (long long)nclusters + 1));
    CCHK(scan_exclusive(ccnt, p->cptr, (long long)nclusters + 1, scr, s));
    // 4. the layout
    int e = layout_alloc(p->clu, n, p->nnz_off);
    if (e) {
        cleanup();
        return e;
    }
    CCHK(dalloc(&pos_of, n));
    k_cluster_rows<<<grid_for((long long)n + 1, 256), 256, 0, s>>>(ord, p->inv, p->lev.ptr, n, p->clu.ptr,
                                                                    p->clu.rowid, pos_of);
    CCHK(cudaGetLastError());
    CCHK(scan_exclusive(p->clu.ptr, p->clu.ptr, (long long)n + 1, scr, s));
    k_cluster_fill<<<grid_for((long long)n * 32, 256), 256, 0, s>>>(p->lev, p->inv, p->clu, cl, pos_of, p->cptr, n);
    CCHK(cudaGetLastError());
    CCHK(cudaStreamSynchronize(s));
#undef CCHK
    p->clu_key = key2;  // sorted: cluster * H + local level per position
    key2 = nullptr;
    cleanup();
    p->nclusters = nclusters;
    p->clu_H = H;
    p->clu_B = B;
    return 0;
}

}  // namespace sptrsv
