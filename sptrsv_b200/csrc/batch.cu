// batch.cu — many independent triangular systems, each with its own number
// of right-hand sides (1..32), solved in one persistent launch.
//
// The union of the systems is one block-diagonal lower-triangular matrix.
// One analysis of the union gives every row its level; the rows are laid out
// in (level, right-hand-side class) order, where the class of a system with
// k right-hand sides is kp = the power of two >= k, and cut into
// level-aligned tasks of 32/kp rows (lane j of a row's kp lanes owns
// right-hand side j).  Tasks are in a topological order of the union, so the
// persistent grid's static round-robin over tasks is deadlock-free and all
// systems advance together: a shallow system finishes early, a deep one
// keeps a few warps busy to the end.
//
// Vectors are packed: system s owns the row-major n_s x k_s block starting at
// element off_s (off_0 = 0, off_{s+1} = off_s + n_s k_s).  Each stored
// off-diagonal entry keeps the packed offset of its column's row, so a wait
// is a single load.
//
// HBM layout (positions p in task order, m off-diagonal entries):
//   ptr[n+1] int32, xrow[n] int64 (packed offset of the row), krow[n] int32,
//   xdep[m] int64 (packed offset of the column's row), val64[m] f64,
//   val32[m] f32, dg64[n] f64, di64[n] f64 (1/diag), di32[n] f32,
//   tbase[ntasks+1], tkp[ntasks].
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"

namespace sptrsv {
int run_analysis_impl(dfr_analysis_info_t* info, const sp_mat_t* L, MODE mode);
}

struct sptrsv_batch_s {
    int nsys = 0;
    int n = 0, nnz = 0, m = 0, nlevs = 0;
    long long nvec = 0;  // packed vector length
    std::vector<long long> off;
    std::vector<int> kk;
    int* ptr = nullptr;
    long long* xrow = nullptr;
    int* krow = nullptr;
    long long* xdep = nullptr;
    double* val64 = nullptr;
    float* val32 = nullptr;
    double* dg64 = nullptr;
    double* di64 = nullptr;
    float* di32 = nullptr;
    int* tbase = nullptr;
    int* tkp = nullptr;
    int ntasks = 0;
    float* w32a = nullptr;
    float* w32b = nullptr;
    // natural-order chunk schedule: the union CSR without its diagonal
    int* nptr = nullptr;         // [n+1] off-diagonal offsets per union row
    int* ncol = nullptr;         // [m] union column
    double* nval64 = nullptr;
    float* nval32 = nullptr;
    double* ndg64 = nullptr;
    double* ndi64 = nullptr;
    float* ndi32 = nullptr;
    int* tsys = nullptr;         // [nchunks] per task: system (tasks in (chunk, system) order)
    int* tj = nullptr;           // [nchunks] per task: chunk index inside its system
    int* cdep = nullptr;         // [nchunks] per task: first chunk of the same system it reads
    int* sys_row0 = nullptr;     // [nsys] first union row
    int* sys_chunk0 = nullptr;   // [nsys] first flag of the system
    int* sys_k = nullptr;        // [nsys]
    long long* sys_off = nullptr;  // [nsys]
    int* flags = nullptr;        // [nchunks] chunk done flags (1 = done)
    int* row_sys = nullptr;      // [n] system of each union row
    int nchunks = 0;
    int chunked = 0;             // 0: level-ordered tasks (default), 1: natural-order chunks
    int block_warps = 8, warps_per_sm = 0, backoff_ns = 0, ir_iters = 2;
    // graph cache for one (b, x, precision)
    cudaGraphExec_t gexec = nullptr;
    const double* g_b = nullptr;
    double* g_x = nullptr;
    int g_prec = 0;
    cudaStream_t cap_stream = nullptr;
};

namespace sptrsv {

namespace {

struct BatchMat {
    const int* __restrict__ ptr;
    const long long* __restrict__ xrow;
    const int* __restrict__ krow;
    const long long* __restrict__ xdep;
};

// variable right-hand-side count, one lane per (row, right-hand side)
template <typename V, typename T, typename BT, int OUT>
__global__ void __launch_bounds__(512) k_sptrsv_vk(BatchMat bm, const V* __restrict__ val, const V* __restrict__ di,
                                                   int ntasks, const int* __restrict__ tbase,
                                                   const int* __restrict__ tkp, const BT* __restrict__ b, T* x,
                                                   double* x64, DevStatus* st, unsigned long long budget,
                                                   unsigned backoff)
{
    const int lane = threadIdx.x & 31;
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    for (int t = gw; t < ntasks; t += nw) {
        const int base = __ldg(tbase + t), cnt = __ldg(tbase + t + 1) - base, kp = __ldg(tkp + t);
        const int seg = lane / kp, k = lane & (kp - 1);
        const int pos = base + seg;
        const bool act = seg < cnt && k < __ldg(bm.krow + (seg < cnt ? pos : base));
        long long xr = 0;
        T acc = 0, piv = 0;
        int s = 0, len = 0;
        if (act) {
            xr = __ldg(bm.xrow + pos);
            acc = (T)b[xr + k];
            piv = (T)__ldg(di + pos);
            s = __ldg(bm.ptr + pos);
            len = __ldg(bm.ptr + pos + 1) - s;
        }
        // rows of a task are in one level: the warp waits for each round together
        const int rounds = __reduce_max_sync(0xffffffffu, len);
        for (int j = 0; j < rounds; j++) {
            const bool have = j < len;
            long long xc = 0;
            T v = 0, xv = 0;
            if (have) {
                xc = __ldg(bm.xdep + s + j);
                v = (T)__ldg(val + s + j);
            }
            if (!warp_wait<false, T>(have, 0, x + xc + k, nullptr, xv, st, budget, backoff, pos)) return;
            if (have) acc -= v * xv;
        }
        if (act) {
            T r = publishable(acc * piv);
            st_relaxed(x + xr + k, r);
            if (OUT == 1) x64[xr + k] = (double)r;
            if (OUT == 2) x64[xr + k] += (double)r;
        }
    }
}

// Natural-order chunk schedule.  Task t is chunk j of system s: its rows
// [row0_s + 32j, +32), solved one after another by one warp, lane q owning
// right-hand side q.  Before its first row the warp waits (warp-convergent,
// acquire) for the done flags of the chunks of the same system that the
// chunk reads (cdep[t] .. j-1); after that every outside value is final.
// Values of earlier rows of the chunk come from the warp's shared-memory
// ring.  When the chunk is done the warp releases its flag.
struct NatBatch {
    const int* __restrict__ ptr;
    const int* __restrict__ col;
    const int* __restrict__ tsys;
    const int* __restrict__ tj;
    const int* __restrict__ cdep;
    const int* __restrict__ row0;
    const int* __restrict__ chunk0;
    const int* __restrict__ sk;
    const long long* __restrict__ soff;
};

template <typename V, typename T, typename BT, int OUT>
__global__ void __launch_bounds__(256) k_sptrsv_vkc(NatBatch nb, const V* __restrict__ val, const V* __restrict__ di,
                                                    int ntasks, int* flags, const BT* __restrict__ b, T* x,
                                                    double* x64, DevStatus* st, unsigned long long budget,
                                                    unsigned backoff)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    T* ring = reinterpret_cast<T*>(smem_raw) + (threadIdx.x >> 5) * 32 * 32;  // [row][rhs]
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    for (int t = gw; t < ntasks; t += nw) {
        const int s = __ldg(nb.tsys + t), j = __ldg(nb.tj + t);
        const int row0 = __ldg(nb.row0 + s), c0 = __ldg(nb.chunk0 + s), K = __ldg(nb.sk + s);
        const long long off = __ldg(nb.soff + s);
        const int nrows_s = __ldg(nb.row0 + s + 1) - row0;
        const int r0 = row0 + 32 * j, cnt = min(32, row0 + nrows_s - r0);
        // wait for the chunks this one reads
        for (int q = __ldg(nb.cdep + t) + lane; __any_sync(0xffffffffu, q < j); q += 32) {
            int fv = 1;
            if (!warp_wait<false, int>(q < j, c0 + q, flags, nullptr, fv, st, budget, backoff, r0)) return;
        }
        __threadfence();  // acquire: the flagged chunks' x values are visible
        const bool lk = lane < K;
        for (int i = 0; i < cnt; i++) {
            const int r = r0 + i;
            const long long xr = off + (long long)(r - row0) * K;
            T acc = lk ? (T)b[xr + lane] : (T)0;
            const T piv = (T)__ldg(di + r);
            const int e0 = __ldg(nb.ptr + r), e1 = __ldg(nb.ptr + r + 1);
            for (int p0 = e0; p0 < e1; p0 += 32) {
                const int nq = min(32, e1 - p0);
                int c = 0;
                T v = 0;
                if (lane < nq) {
                    c = __ldg(nb.col + p0 + lane);
                    v = (T)__ldg(val + p0 + lane);
                }
#pragma unroll 4
                for (int u = 0; u < nq; u++) {
                    const int cu = __shfl_sync(0xffffffffu, c, u);
                    const T vu = __shfl_sync(0xffffffffu, v, u);
                    T xv = 0;
                    if (lk) xv = cu >= r0 ? ring[(cu - r0) * 32 + lane] : ld_relaxed(x + off + (long long)(cu - row0) * K + lane);
                    acc -= vu * xv;
                }
            }
            if (lk) {
                const T res = publishable(acc * piv);
                ring[i * 32 + lane] = res;
                st_relaxed(x + xr + lane, res);
                if (OUT == 1) x64[xr + lane] = (double)res;
                if (OUT == 2) x64[xr + lane] += (double)res;
            }
            __syncwarp();
        }
        __threadfence();  // release: this chunk's x values before its flag
        if (lane == 0) st_relaxed(flags + c0 + j, 1);
    }
}

// r = b - L x in FP64 over the natural-order union, one warp per row, lanes over the right-hand sides
__global__ void __launch_bounds__(256) k_residual_vkc(const int* __restrict__ ptr, const int* __restrict__ col,
                                                      const double* __restrict__ val, const double* __restrict__ dg,
                                                      const int* __restrict__ row_sys, const int* __restrict__ row0,
                                                      const int* __restrict__ sk, const long long* __restrict__ soff,
                                                      int n, const double* __restrict__ b,
                                                      const double* __restrict__ x, float* __restrict__ r)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const int s = row_sys[i], K = sk[s], r0 = row0[s];
        if (lane >= K) continue;
        const long long o = soff[s];
        const long long xr = o + (long long)(i - r0) * K + lane;
        double acc = b[xr] - dg[i] * x[xr];
        for (int p = ptr[i]; p < ptr[i + 1]; p++) acc -= val[p] * x[o + (long long)(col[p] - r0) * K + lane];
        r[xr] = (float)acc;
    }
}

// r = b - L x in FP64 over the batch layout (no dependencies)
__global__ void __launch_bounds__(256) k_residual_vk(BatchMat bm, const double* __restrict__ val,
                                                     const double* __restrict__ dg, int ntasks,
                                                     const int* __restrict__ tbase, const int* __restrict__ tkp,
                                                     const double* __restrict__ b, const double* __restrict__ x,
                                                     float* __restrict__ r)
{
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long t = gw; t < ntasks; t += nw) {
        const int base = tbase[t], cnt = tbase[t + 1] - base, kp = tkp[t];
        const int seg = lane / kp, k = lane & (kp - 1);
        if (seg >= cnt) continue;
        const int pos = base + seg;
        if (k >= bm.krow[pos]) continue;
        const long long xr = bm.xrow[pos];
        double acc = b[xr + k] - dg[pos] * x[xr + k];
        for (int p = bm.ptr[pos]; p < bm.ptr[pos + 1]; p++) acc -= val[p] * x[bm.xdep[p] + k];
        r[xr + k] = (float)acc;
    }
}

// ---- build ----
__global__ void k_union_rows(const int* __restrict__ rp, int n_s, int row0, int nnz0, int* __restrict__ urp)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_s; i += gridDim.x * blockDim.x)
        urp[row0 + i] = nnz0 + rp[i];
}
__global__ void k_union_cols(const int* __restrict__ ci, int nnz_s, int row0, int* __restrict__ uci)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz_s; i += gridDim.x * blockDim.x) uci[i] = ci[i] + row0;
}

// key = (level-1)*6 + log2(kp) per union row; row data for the layout
__global__ void k_batch_keys(const int* __restrict__ level, const int* __restrict__ sys_of_row,
                             const int* __restrict__ kp_log, int n, int* __restrict__ key, int* __restrict__ iota)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        key[i] = (level[i] - 1) * 6 + kp_log[sys_of_row[i]];
        iota[i] = i;
    }
}

__global__ void k_batch_rows(const int* __restrict__ order, const int* __restrict__ urp, int n,
                             int* __restrict__ len, int* __restrict__ pos_of)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= n; p += gridDim.x * blockDim.x) {
        if (p == n) {
            len[p] = 0;
            continue;
        }
        int r = order[p];
        pos_of[r] = p;
        len[p] = urp[r + 1] - urp[r] - 1;
    }
}

__global__ void k_batch_fill(const int* __restrict__ order, const int* __restrict__ urp, const int* __restrict__ uci,
                             const double* __restrict__ uva, const int* __restrict__ sys_of_row,
                             const int* __restrict__ row0, const long long* __restrict__ soff,
                             const int* __restrict__ sk, const int* __restrict__ ptr, int n, long long* __restrict__ xrow,
                             int* __restrict__ krow, long long* __restrict__ xdep, double* __restrict__ val64,
                             float* __restrict__ val32, double* __restrict__ dg64, double* __restrict__ di64,
                             float* __restrict__ di32)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n; p += nw) {
        const int r = order[p];
        const int s = sys_of_row[r];
        const long long o = soff[s];
        const int k = sk[s], r0 = row0[s];
        const int a = urp[r], e = urp[r + 1] - 1, dst = ptr[p];
        for (int q = a + lane; q < e; q += 32) {
            const int c = uci[q];
            xdep[dst + q - a] = o + (long long)(c - r0) * k;
            val64[dst + q - a] = uva[q];
            val32[dst + q - a] = (float)uva[q];
        }
        if (lane == 0) {
            const double d = uva[e];
            xrow[p] = o + (long long)(r - r0) * k;
            krow[p] = k;
            dg64[p] = d;
            di64[p] = 1.0 / d;
            di32[p] = 1.0f / (float)d;
        }
    }
}

// natural-order union without diagonals: nptr[i] = ia[i] - i (one diagonal per earlier row)
__global__ void k_nat_fill(const int* __restrict__ urp, const int* __restrict__ uci, const double* __restrict__ uva,
                           int n, int* __restrict__ nptr, int* __restrict__ ncol, double* __restrict__ nval64,
                           float* __restrict__ nval32, double* __restrict__ ndg, double* __restrict__ ndi,
                           float* __restrict__ ndi32)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const int a = urp[i], e = urp[i + 1] - 1, o = a - (int)i;
        for (int q = a + lane; q < e; q += 32) {
            ncol[o + q - a] = uci[q];
            nval64[o + q - a] = uva[q];
            nval32[o + q - a] = (float)uva[q];
        }
        if (lane == 0) {
            const double d = uva[e];
            nptr[i] = o;
            ndg[i] = d;
            ndi[i] = 1.0 / d;
            ndi32[i] = 1.0f / (float)d;
            if (i == n - 1) nptr[n] = e - (int)i;
        }
    }
}

// first chunk each natural chunk reads: the chunk of its smallest column
__global__ void k_chunk_dep(const int* __restrict__ nptr, const int* __restrict__ ncol,
                            const int* __restrict__ chunk0, const int* __restrict__ row0, int nsys, int nchunks,
                            int* __restrict__ dep)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        int lo = 0, hi = nsys - 1;  // system: largest s with chunk0[s] <= c
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (chunk0[mid] <= c) lo = mid;
            else hi = mid - 1;
        }
        const int s = lo, j = c - chunk0[s];
        const int r0 = row0[s] + 32 * j, r1 = min(r0 + 32, row0[s + 1]);
        int mn = r0;
        for (int r = r0; r < r1; r++)
            if (nptr[r + 1] > nptr[r]) mn = min(mn, ncol[nptr[r]]);
        dep[c] = (mn - row0[s]) / 32;
    }
}

__global__ void k_task_kp(const int* __restrict__ tbase, int ntasks, const int* __restrict__ key_sorted,
                          int* __restrict__ tkp)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x)
        tkp[t] = 1 << (key_sorted[tbase[t]] % 6);
}

void batch_free(sptrsv_batch_s* B)
{
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    if (B->cap_stream) cudaStreamDestroy(B->cap_stream);
    cudaFree(B->nptr); cudaFree(B->ncol); cudaFree(B->nval64); cudaFree(B->nval32); cudaFree(B->ndg64);
    cudaFree(B->ndi64); cudaFree(B->ndi32); cudaFree(B->tsys); cudaFree(B->tj); cudaFree(B->cdep);
    cudaFree(B->sys_row0); cudaFree(B->sys_chunk0); cudaFree(B->sys_k); cudaFree(B->sys_off); cudaFree(B->flags);
    cudaFree(B->row_sys);
    cudaFree(B->ptr); cudaFree(B->xrow); cudaFree(B->krow); cudaFree(B->xdep); cudaFree(B->val64);
    cudaFree(B->val32); cudaFree(B->dg64); cudaFree(B->di64); cudaFree(B->di32); cudaFree(B->tbase);
    cudaFree(B->tkp); cudaFree(B->w32a); cudaFree(B->w32b);
}

// Level- and class-aligned tasks: a segment is one (level, kp) key and is
// cut into tasks of 32/kp rows; tkp[t] = kp of the task's segment.
int batch_tasks(sptrsv_batch_s* B, const int* key_sorted, int K, cudaStream_t s)
{
    int e = build_task_table(key_sorted, B->n, K, 0, &B->tbase, &B->ntasks, s);
    if (e) return e;
    SPT_CUDA(dalloc(&B->tkp, B->ntasks));
    if (B->ntasks > 0) {
        k_task_kp<<<grid_for(B->ntasks, 256), 256, 0, s>>>(B->tbase, B->ntasks, key_sorted, B->tkp);
        SPT_CUDA(cudaGetLastError());
    }
    return 0;
}

template <typename V, typename T, typename BT, int OUT>
int batch_launch(sptrsv_batch_s* B, bool f32, const BT* b, T* x, double* x64, cudaStream_t s)
{
    Ctx* c = ctx();
    const int block = 32 * B->block_warps;
    const int cap = B->warps_per_sm > 0 ? (B->warps_per_sm + B->block_warps - 1) / B->block_warps : 0;
    if (B->chunked) {
        const V* val = f32 ? reinterpret_cast<const V*>(B->nval32) : reinterpret_cast<const V*>(B->nval64);
        const V* di = f32 ? reinterpret_cast<const V*>(B->ndi32) : reinterpret_cast<const V*>(B->ndi64);
        NatBatch nb{B->nptr, B->ncol, B->tsys, B->tj, B->cdep, B->sys_row0, B->sys_chunk0, B->sys_k, B->sys_off};
        SPT_CUDA(cudaMemsetAsync(B->flags, 0, sizeof(int) * (size_t)B->nchunks, s));
        auto kern = k_sptrsv_vkc<V, T, BT, OUT>;
        const size_t smem = (size_t)B->block_warps * 32 * 32 * sizeof(T);
        if (smem > 48 * 1024)
            SPT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        SPT_CUDA(launch_persistent_capped(kern, block, smem, div_up(B->nchunks, B->block_warps), cap, s, nb, val, di,
                                          B->nchunks, B->flags, b, x, x64, c->d_status, wait_budget_ns(),
                                          (unsigned)B->backoff_ns));
        return 0;
    }
    const V* val = f32 ? reinterpret_cast<const V*>(B->val32) : reinterpret_cast<const V*>(B->val64);
    const V* di = f32 ? reinterpret_cast<const V*>(B->di32) : reinterpret_cast<const V*>(B->di64);
    BatchMat bm{B->ptr, B->xrow, B->krow, B->xdep};
    auto kern = k_sptrsv_vk<V, T, BT, OUT>;
    SPT_CUDA(launch_persistent_capped(kern, block, 0, div_up(B->ntasks, B->block_warps), cap, s, bm, val, di,
                                      B->ntasks, (const int*)B->tbase, (const int*)B->tkp, b, x, x64, c->d_status,
                                      wait_budget_ns(), (unsigned)B->backoff_ns));
    return 0;
}

int batch_residual(sptrsv_batch_s* B, const double* b, const double* x, cudaStream_t s)
{
    if (B->chunked) {
        k_residual_vkc<<<grid_for((long long)B->n * 32, 256), 256, 0, s>>>(B->nptr, B->ncol, B->nval64, B->ndg64,
                                                                          B->row_sys, B->sys_row0, B->sys_k,
                                                                          B->sys_off, B->n, b, x, B->w32b);
    } else {
        BatchMat bm{B->ptr, B->xrow, B->krow, B->xdep};
        k_residual_vk<<<grid_for((long long)B->ntasks * 32, 256), 256, 0, s>>>(bm, B->val64, B->dg64, B->ntasks,
                                                                                B->tbase, B->tkp, b, x, B->w32b);
    }
    SPT_CUDA(cudaGetLastError());
    return 0;
}

int batch_solve_impl(sptrsv_batch_s* B, const double* b, double* x, int precision, cudaStream_t s)
{
    if (B->n == 0) return 0;
    if (precision == 64) {
        SPT_CUDA(cudaMemsetAsync(x, 0xFF, sizeof(double) * (size_t)B->nvec, s));
        return batch_launch<double, double, double, 0>(B, false, b, x, nullptr, s);
    }
    const size_t b32 = sizeof(float) * (size_t)B->nvec;
    SPT_CUDA(cudaMemsetAsync(B->w32a, 0xFF, b32, s));
    int e = batch_launch<float, float, double, 1>(B, true, b, B->w32a, x, s);
    if (e) return e;
    for (int it = 0; it < B->ir_iters; it++) {
        e = batch_residual(B, b, x, s);
        if (e) return e;
        SPT_CUDA(cudaMemsetAsync(B->w32a, 0xFF, b32, s));
        e = batch_launch<float, float, float, 2>(B, true, B->w32b, B->w32a, x, s);
        if (e) return e;
    }
    return 0;
}

}  // namespace

}  // namespace sptrsv

using namespace sptrsv;

extern "C" {

int sptrsv_batch_create(int nsys, const sp_mat_t* mats, const int* nrhs, sptrsv_batch_t* out)
{
    if (!out || nsys < 1 || !mats || !nrhs) return set_error(SPTRSV_ERR_INVALID_ARG, "batch_create: bad arguments");
    *out = nullptr;
    Ctx* c = ctx();
    if (!c) return set_error(SPTRSV_ERR_CUDA, "batch_create: no CUDA device");
    long long n = 0, nnz = 0, nvec = 0;
    for (int s = 0; s < nsys; s++) {
        if (nrhs[s] < 1 || nrhs[s] > 32 || mats[s].nr < 1 || mats[s].nc != mats[s].nr || mats[s].nnz < mats[s].nr)
            return set_error(SPTRSV_ERR_INVALID_ARG, "batch_create: system %d: bad sizes or nrhs", s);
        n += mats[s].nr;
        nnz += mats[s].nnz;
        nvec += (long long)mats[s].nr * nrhs[s];
    }
    if (n > 0x7fffffffLL || nnz > 0x7fffffffLL) return set_error(SPTRSV_ERR_UNSUPPORTED, "batch_create: union too large");
    sptrsv_batch_s* B = new sptrsv_batch_s();
    B->nsys = nsys;
    B->n = (int)n;
    B->nnz = (int)nnz;
    B->m = (int)(nnz - n);
    B->nvec = nvec;
    B->off.resize(nsys + 1);
    B->kk.assign(nrhs, nrhs + nsys);
    std::vector<int> row0(nsys + 1), kplog(nsys), sys_of_row((size_t)n);
    B->off[0] = 0;
    row0[0] = 0;
    for (int s = 0; s < nsys; s++) {
        B->off[s + 1] = B->off[s] + (long long)mats[s].nr * nrhs[s];
        row0[s + 1] = row0[s] + mats[s].nr;
        int j = 0;
        while ((1 << j) < nrhs[s]) j++;
        kplog[s] = j;
        std::fill(sys_of_row.begin() + row0[s], sys_of_row.begin() + row0[s + 1], s);
    }
    // device scratch
    sp_mat_t U{};
    dfr_analysis_info_t info{};
    int *d_sys = nullptr, *d_row0 = nullptr, *d_kplog = nullptr, *d_sk = nullptr, *key = nullptr, *ord = nullptr;
    int *kt = nullptr, *vt = nullptr, *scr = nullptr, *pos_of = nullptr;
    long long* d_soff = nullptr;
    auto cleanup = [&]() {
        cudaFree(U.ia); cudaFree(U.ja); cudaFree(U.a);
        cudaFree(d_sys); cudaFree(d_row0); cudaFree(d_kplog); cudaFree(d_sk); cudaFree(d_soff);
        cudaFree(key); cudaFree(ord); cudaFree(kt); cudaFree(vt); cudaFree(scr); cudaFree(pos_of);
    };
    auto fail = [&](int code) {
        cleanup();
        free_device_analysis(nullptr, &info);
        batch_free(B);
        delete B;
        return code;
    };
#define BCHK(call)                                                 \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, #call));  \
    } while (0)
    cudaStream_t s = 0;
    // 1. union CSR
    BCHK(dalloc(&U.ia, n + 1));
    BCHK(dalloc(&U.ja, nnz));
    BCHK(dalloc(&U.a, nnz));
    {
        long long nz0 = 0;
        for (int k = 0; k < nsys; k++) {
            k_union_rows<<<grid_for(mats[k].nr, 256), 256, 0, s>>>(mats[k].ia, mats[k].nr, row0[k], (int)nz0, U.ia);
            k_union_cols<<<grid_for(mats[k].nnz, 256), 256, 0, s>>>(mats[k].ja, mats[k].nnz, row0[k], U.ja + nz0);
            BCHK(cudaMemcpyAsync(U.a + nz0, mats[k].a, sizeof(double) * (size_t)mats[k].nnz, cudaMemcpyDeviceToDevice, s));
            nz0 += mats[k].nnz;
        }
        int last = (int)nnz;
        BCHK(cudaMemcpyAsync(U.ia + n, &last, sizeof(int), cudaMemcpyHostToDevice, s));
        BCHK(cudaGetLastError());
        BCHK(cudaStreamSynchronize(s));
    }
    U.nr = U.nc = (int)n;
    U.nnz = (int)nnz;
    // 2. levels of the union (validates every system's CSR too)
    {
        int e = run_analysis_impl(&info, &U, ORDER);
        if (e) return fail(e);
    }
    AnalysisRec* rec = find_analysis(info.row_ctr);
    B->nlevs = info.nlevs;
    // 3. order (level, rhs class), stable in the natural order
    BCHK(dalloc(&d_sys, n));
    BCHK(dalloc(&d_row0, nsys + 1));
    BCHK(dalloc(&d_kplog, nsys));
    BCHK(dalloc(&d_sk, nsys));
    BCHK(dalloc(&d_soff, nsys + 1));
    BCHK(cudaMemcpy(d_sys, sys_of_row.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    BCHK(cudaMemcpy(d_row0, row0.data(), sizeof(int) * (size_t)(nsys + 1), cudaMemcpyHostToDevice));
    BCHK(cudaMemcpy(d_kplog, kplog.data(), sizeof(int) * (size_t)nsys, cudaMemcpyHostToDevice));
    BCHK(cudaMemcpy(d_sk, nrhs, sizeof(int) * (size_t)nsys, cudaMemcpyHostToDevice));
    BCHK(cudaMemcpy(d_soff, B->off.data(), sizeof(long long) * (size_t)(nsys + 1), cudaMemcpyHostToDevice));
    BCHK(dalloc(&key, n));
    BCHK(dalloc(&ord, n));
    BCHK(dalloc(&kt, n));
    BCHK(dalloc(&vt, n));
    long long sc1 = radix_scratch_ints(n), sc2 = scan_scratch_ints(n + 1);
    BCHK(dalloc(&scr, sc1 > sc2 ? sc1 : sc2));
    k_batch_keys<<<grid_for(n, 256), 256, 0, s>>>(rec->d_levels, d_sys, d_kplog, (int)n, key, ord);
    BCHK(cudaGetLastError());
    BCHK(radix_sort_pairs(key, ord, kt, vt, n, 6 * info.nlevs - 1, scr, s));
    // 4. layout
    BCHK(dalloc(&B->ptr, n + 1));
    BCHK(dalloc(&pos_of, n));
    k_batch_rows<<<grid_for(n + 1, 256), 256, 0, s>>>(ord, U.ia, (int)n, B->ptr, pos_of);
    BCHK(cudaGetLastError());
    BCHK(scan_exclusive(B->ptr, B->ptr, n + 1, scr, s));
    BCHK(dalloc(&B->xrow, n));
    BCHK(dalloc(&B->krow, n));
    BCHK(dalloc(&B->xdep, B->m));
    BCHK(dalloc(&B->val64, B->m));
    BCHK(dalloc(&B->val32, B->m));
    BCHK(dalloc(&B->dg64, n));
    BCHK(dalloc(&B->di64, n));
    BCHK(dalloc(&B->di32, n));
    k_batch_fill<<<grid_for(n * 32, 256), 256, 0, s>>>(ord, U.ia, U.ja, U.a, d_sys, d_row0, d_soff, d_sk, B->ptr,
                                                        (int)n, B->xrow, B->krow, B->xdep, B->val64, B->val32,
                                                        B->dg64, B->di64, B->di32);
    BCHK(cudaGetLastError());
    {
        int e = batch_tasks(B, key, 6 * info.nlevs, s);
        if (e) return fail(e);
    }
    // 5. natural-order chunk schedule: union without diagonals, chunk tasks in
    //    (chunk index, system) order, each with the first chunk it reads
    BCHK(dalloc(&B->nptr, n + 1));
    BCHK(dalloc(&B->ncol, B->m));
    BCHK(dalloc(&B->nval64, B->m));
    BCHK(dalloc(&B->nval32, B->m));
    BCHK(dalloc(&B->ndg64, n));
    BCHK(dalloc(&B->ndi64, n));
    BCHK(dalloc(&B->ndi32, n));
    k_nat_fill<<<grid_for(n * 32, 256), 256, 0, s>>>(U.ia, U.ja, U.a, (int)n, B->nptr, B->ncol, B->nval64, B->nval32,
                                                      B->ndg64, B->ndi64, B->ndi32);
    BCHK(cudaGetLastError());
    {
        std::vector<int> chunk0(nsys + 1), nch(nsys);
        int maxch = 0;
        chunk0[0] = 0;
        for (int k = 0; k < nsys; k++) {
            nch[k] = (mats[k].nr + 31) / 32;
            chunk0[k + 1] = chunk0[k] + nch[k];
            maxch = std::max(maxch, nch[k]);
        }
        B->nchunks = chunk0[nsys];
        BCHK(dalloc(&B->sys_row0, nsys + 1));
        BCHK(dalloc(&B->sys_chunk0, nsys + 1));
        BCHK(dalloc(&B->sys_k, nsys));
        BCHK(dalloc(&B->sys_off, nsys + 1));
        BCHK(cudaMemcpy(B->sys_row0, row0.data(), sizeof(int) * (size_t)(nsys + 1), cudaMemcpyHostToDevice));
        BCHK(cudaMemcpy(B->sys_chunk0, chunk0.data(), sizeof(int) * (size_t)(nsys + 1), cudaMemcpyHostToDevice));
        BCHK(cudaMemcpy(B->sys_k, nrhs, sizeof(int) * (size_t)nsys, cudaMemcpyHostToDevice));
        BCHK(cudaMemcpy(B->sys_off, B->off.data(), sizeof(long long) * (size_t)(nsys + 1), cudaMemcpyHostToDevice));
        int* dep_nat = nullptr;
        BCHK(dalloc(&dep_nat, B->nchunks));
        k_chunk_dep<<<grid_for(B->nchunks, 256), 256, 0, s>>>(B->nptr, B->ncol, B->sys_chunk0, B->sys_row0, nsys,
                                                               B->nchunks, dep_nat);
        std::vector<int> dn(B->nchunks);
        cudaError_t ce = cudaMemcpy(dn.data(), dep_nat, sizeof(int) * (size_t)B->nchunks, cudaMemcpyDeviceToHost);
        cudaFree(dep_nat);
        BCHK(ce);
        std::vector<int> ts, tjv, td;
        ts.reserve(B->nchunks);
        tjv.reserve(B->nchunks);
        td.reserve(B->nchunks);
        for (int j = 0; j < maxch; j++)
            for (int k = 0; k < nsys; k++)
                if (j < nch[k]) {
                    ts.push_back(k);
                    tjv.push_back(j);
                    td.push_back(dn[chunk0[k] + j]);
                }
        BCHK(dalloc(&B->tsys, B->nchunks));
        BCHK(dalloc(&B->tj, B->nchunks));
        BCHK(dalloc(&B->cdep, B->nchunks));
        BCHK(dalloc(&B->flags, B->nchunks));
        BCHK(cudaMemcpy(B->tsys, ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice));
        BCHK(cudaMemcpy(B->tj, tjv.data(), sizeof(int) * tjv.size(), cudaMemcpyHostToDevice));
        BCHK(cudaMemcpy(B->cdep, td.data(), sizeof(int) * td.size(), cudaMemcpyHostToDevice));
    }
    B->row_sys = d_sys;  // kept for the natural-order residual
    d_sys = nullptr;
    BCHK(dalloc(&B->w32a, B->nvec));
    BCHK(dalloc(&B->w32b, B->nvec));
    BCHK(cudaStreamSynchronize(s));
#undef BCHK
    cleanup();
    free_device_analysis(nullptr, &info);
    *out = B;
    return ok();
}

int sptrsv_batch_destroy(sptrsv_batch_t B)
{
    if (!B) return ok();
    batch_free(B);
    delete B;
    return ok();
}

int sptrsv_batch_info(sptrsv_batch_t B, long long* offsets, int* n_total, int* nlevs, long long* vec_len)
{
    if (!B) return set_error(SPTRSV_ERR_INVALID_ARG, "batch_info: NULL");
    if (offsets) memcpy(offsets, B->off.data(), sizeof(long long) * (size_t)(B->nsys + 1));
    if (n_total) *n_total = B->n;
    if (nlevs) *nlevs = B->nlevs;
    if (vec_len) *vec_len = B->nvec;
    return ok();
}

int sptrsv_batch_set_schedule(sptrsv_batch_t B, int chunked, int block_warps, int warps_per_sm, int backoff_ns,
                              int ir_iters)
{
    if (!B || (chunked != 0 && chunked != 1) ||
        (block_warps != 2 && block_warps != 4 && block_warps != 8 && block_warps != 16) ||
        (chunked && block_warps > 8) || warps_per_sm < 0 || warps_per_sm > 64 || backoff_ns < 0 ||
        backoff_ns > 100000 || ir_iters < 0 || ir_iters > 16)
        return set_error(SPTRSV_ERR_INVALID_ARG, "batch_set_schedule: bad arguments");
    B->chunked = chunked;
    B->block_warps = block_warps;
    B->warps_per_sm = warps_per_sm;
    B->backoff_ns = backoff_ns;
    B->ir_iters = ir_iters;
    if (B->gexec) {  // the captured graph encodes the old schedule
        cudaGraphExecDestroy(B->gexec);
        B->gexec = nullptr;
    }
    return ok();
}

int sptrsv_batch_solve(sptrsv_batch_t B, const double* b, double* x, int precision, cudaStream_t s)
{
    if (!B || !b || !x || (precision != 32 && precision != 64))
        return set_error(SPTRSV_ERR_INVALID_ARG, "batch_solve: bad arguments");
    int e = batch_solve_impl(B, b, x, precision, s);
    return e ? e : ok();
}

// Captures the whole solve (memsets, persistent solve launches, residuals) as
// a CUDA graph on first use for these (b, x, precision) and replays it on
// `s`; a different (b, x, precision) re-captures.
int sptrsv_batch_solve_graph(sptrsv_batch_t B, const double* b, double* x, int precision, cudaStream_t s)
{
    if (!B || !b || !x || (precision != 32 && precision != 64))
        return set_error(SPTRSV_ERR_INVALID_ARG, "batch_solve_graph: bad arguments");
    if (!B->gexec || B->g_b != b || B->g_x != x || B->g_prec != precision) {
        if (B->gexec) {
            cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
        }
        if (!B->cap_stream) SPT_CUDA(cudaStreamCreateWithFlags(&B->cap_stream, cudaStreamNonBlocking));
        // make sure everything the capture reads (occupancy caches, context) exists
        ctx();
        cudaGraph_t g = nullptr;
        SPT_CUDA(cudaStreamBeginCapture(B->cap_stream, cudaStreamCaptureModeThreadLocal));
        int e = batch_solve_impl(B, b, x, precision, B->cap_stream);
        cudaError_t ce = cudaStreamEndCapture(B->cap_stream, &g);
        if (e) {
            if (g) cudaGraphDestroy(g);
            return e;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "batch graph capture");
        ce = cudaGraphInstantiate(&B->gexec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            B->gexec = nullptr;
            return cuda_fail(ce, "batch graph instantiate");
        }
        B->g_b = b;
        B->g_x = x;
        B->g_prec = precision;
    }
    SPT_CUDA(cudaGraphLaunch(B->gexec, s));
    return ok();
}

}  // extern "C"
