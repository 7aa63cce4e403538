// solve.cu — host side of the solves: the reference entry points
// (header/solver.h:5-7) over the caller's CSR, and the plan API over the
// plan's layouts (FP64, FP32 + FP64 refinement, 1-32 RHS).
#include <algorithm>
#include <cstring>

#include "internal.h"
#include "plan.h"
#include "solve_kernels.cuh"

namespace sptrsv {

namespace {

constexpr int kRefBlock = 256;  // block of the reference-named solves
constexpr int kRefWarps = kRefBlock / 32;

bool pow2_lanes(int l) { return l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32; }

// Rows of one WAVE line group: their FP64 x values fill the CTA's shared memory.
constexpr int kWaveMaxRows = 200 * 1024 / 8;
// Streamed host solves: rows per copied segment of b, by default an eighth
// of the rows but at least 131072 (1 MiB of doubles), a multiple of 16 rows
// so no 128-byte line of b spans two segments; sptrsv_plan_set_stream_segment
// sets a plan's own.  Every segment costs two queued copies (its rows and its
// flag word), whose fixed cost outweighs an earlier start of the solve: on the
// 2048 x 2048 grid 32 segments took 1.36 ms end to end, 8 segments 1.08 ms.
constexpr int kStreamSegRows = 1 << 17;
int stream_seg_rows(const sptrsv_plan_s* p)
{
    if (p->seg_rows > 0) return p->seg_rows;
    const long long eighth = ((long long)p->n + 7) / 8;
    return (int)std::max<long long>(kStreamSegRows, (eighth + 15) / 16 * 16);
}

// Shared memory of the STRIP kernel: per warp a ring of 2R chunks of 32 values.
size_t strip_smem_bytes(const sptrsv_schedule_t* s, size_t elem)
{
    return (size_t)s->block_warps * 2 * s->rows_per_warp * 32 * elem;
}

__global__ void k_iorder_level_keys(const int* __restrict__ iorder, const int* __restrict__ level, int n,
                                    int* __restrict__ key)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) key[p] = level[iorder[p]] - 1;
}

// Level-aligned tasks over iorder for `lanes` lanes per row, cached with the analysis.
int tile_tasks(AnalysisRec* rec, const int* iorder, int lanes, const int** tasks, int* ntasks)
{
    int j = 0;
    while ((32 >> j) != lanes) j++;
    if (!rec->tile_tasks[j]) {
        int* key = nullptr;
        SPT_CUDA(dalloc(&key, rec->n));
        k_iorder_level_keys<<<grid_for(rec->n, 256), 256>>>(iorder, rec->d_levels, rec->n, key);
        cudaError_t ce = cudaGetLastError();
        int e = ce == cudaSuccess ? build_task_table(key, rec->n, rec->nlevs > 0 ? rec->nlevs : 1, 32 / lanes,
                                                      &rec->tile_tasks[j], &rec->tile_ntasks[j], 0)
                                  : cuda_fail(ce, "tile tasks");
        cudaFree(key);
        if (e) return e;
    }
    *tasks = rec->tile_tasks[j];
    *ntasks = rec->tile_ntasks[j];
    return 0;
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
        SPT_CUDA(launch_persistent(kern, kRefBlock, 0, div_up(nw, kRefWarps), s, m, n, nw, 0, ibase, ivect, b, x,
                                   (double*)nullptr, c->d_status, budget, 0u));
    } else if (mode == ORDER && lanes && lanes < 32) {
        // order with a tile of `lanes` lanes: tasks never cross a level, so the
        // rows of one warp are independent
        AnalysisRec* rec = find_analysis(info->row_ctr);
        if (!rec) return set_error(SPTRSV_ERR_NOT_ANALYSED, "solve: no analysis record for this info");
        const int* tasks = nullptr;
        int ntasks = 0;
        int e = tile_tasks(rec, info->iorder, lanes, &tasks, &ntasks);
        if (e) return e;
        SPT_CUDA(launch_persistent(kern, kRefBlock, 0, div_up(ntasks, kRefWarps), s, m, n, ntasks, lanes, tasks,
                                   (const int*)nullptr, b, x, (double*)nullptr, c->d_status, budget, 0u));
    } else if (mode == ORDER) {
        // one row per warp, in iorder (solve_csr_order.cu:83-149)
        SPT_CUDA(launch_persistent(kern, kRefBlock, 0, div_up(n, kRefWarps), s, m, n, n, 32, (const int*)nullptr,
                                   (const int*)nullptr, b, x, (double*)nullptr, c->d_status, budget, 0u));
    } else {
        // SIMPLE (solve_csr_simple.cu:10-108) walks the natural order in
        // chunks: the reference gives a block a run of rows and resolves
        // dependencies inside the block through shared memory; here a warp
        // takes 32 consecutive rows, solves them in sequence and reads
        // in-chunk dependencies from its shared-memory ring
        auto kc = k_sptrsv_chunk<NatMat, double, double, OUT_X>;
        SPT_CUDA(launch_persistent(kc, kRefBlock, 0, div_up(div_up(n, 32), kRefWarps), s, m, n, 32, b, x,
                                   (double*)nullptr, c->d_status, budget, 0u));
    }
    return ok();
}

// ---- plan ----------------------------------------------------------------------

int plan_solve_f64(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s);

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
__global__ void k_plan_fill(const int* __restrict__ rowptr, const int* __restrict__ col,
                            const double* __restrict__ val, SptLayout l, int n)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long k = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nw) {
        int r = l.rowid[k];
        int s = rowptr[r], e = rowptr[r + 1] - 1, o = l.ptr[k];
        for (int p = s + lane; p < e; p += 32) {
            double v = val[p];
            l.col[o + p - s] = col[p];
            l.val64[o + p - s] = v;
            l.val32[o + p - s] = (float)v;
        }
        if (lane == 0) {
            double d = val[e];
            l.dg64[k] = d;
            l.dg32[k] = (float)d;
            l.di64[k] = 1.0 / d;
            l.di32[k] = 1.0f / (float)d;
        }
    }
}

void plan_free_arrays(sptrsv_plan_s* p)
{
    layout_free(p->lev);
    layout_free(p->clu);
    strip_free(p->strip);
    wave_free(p->wave);
    cudaFree(p->cptr); cudaFree(p->inv); cudaFree(p->levels); cudaFree(p->ibase); cudaFree(p->ivect);
    for (int j = 0; j < 6; j++) {
        cudaFree(p->ord_tasks[j]);
        mrhs_free(p->mrhs[j]);
    }
    cudaFree(p->clu_key); cudaFree(p->clu_tasks); cudaFree(p->clu_ctask);
    cudaFree(p->w32a); cudaFree(p->w32b); cudaFree(p->hb); cudaFree(p->hx);
    cudaFree(p->bflag);
    part_free(p);
    band_free(p->band);
    if (p->epochs) cudaFreeHost(p->epochs);
    if (p->ev_start) cudaEventDestroy(p->ev_start);
    if (p->ev_copied) cudaEventDestroy(p->ev_copied);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
}

// Pinned host memory the device can address directly (its device pointer),
// else nullptr.
void* mapped_host(const void* h)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
    return a.devicePointer;
}

// The streamed host solve of a WAVE plan (FP64, one right-hand side, pinned
// host b and x): b goes to the device in segments on a side stream, each
// segment followed by a 4-byte copy of the call's epoch into its flag word,
// while the solve kernel already runs; the kernel waits for a segment's flag
// before it reads its b, and writes x to the host array as groups of rows
// finish.  The side stream never waits on the kernel; the kernel's waits are
// bounded.
int solve_host_streamed(sptrsv_plan_s* p, const double* hb, double* hx_dev, cudaStream_t s)
{
    const int n = p->n;
    const int seg_rows = stream_seg_rows(p);
    const int nseg = (n + seg_rows - 1) / seg_rows;
    if (!p->bflag || p->nseg < nseg) {
        cudaFree(p->bflag);
        p->bflag = nullptr;
        SPT_CUDA(dalloc(&p->bflag, nseg));
        // zeroed on s, which the copy stream follows (a legacy-stream memset
        // is not ordered before work on a non-blocking stream)
        SPT_CUDA(cudaMemsetAsync(p->bflag, 0, sizeof(int) * (size_t)nseg, s));
        p->nseg = nseg;
    }
    if (!p->epochs) {
        SPT_CUDA(cudaHostAlloc((void**)&p->epochs, sizeof(int) * 256, cudaHostAllocDefault));
        for (int e = 0; e < 256; e++) p->epochs[e] = e;
    }
    if (!p->copy_stream) SPT_CUDA(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    if (!p->ev_start) SPT_CUDA(cudaEventCreateWithFlags(&p->ev_start, cudaEventDisableTiming));
    if (!p->ev_copied) SPT_CUDA(cudaEventCreateWithFlags(&p->ev_copied, cudaEventDisableTiming));
    p->epoch = p->epoch % 255 + 1;  // 1..255: never the flags' initial 0, never the previous call's value
    // the copies overwrite the device b only after everything queued before
    // this call on s; the kernel is queued first (its waits cover the copies),
    // so the time the host spends queueing the copies overlaps the solve
    SPT_CUDA(cudaEventRecord(p->ev_start, s));
    SPT_CUDA(cudaStreamWaitEvent(p->copy_stream, p->ev_start, 0));
    // a partitioned plan streams through its block system: that plan's WAVE
    // layout maps each slot to the outer row of its b and each group to the
    // outer rows of its real rows
    sptrsv_plan_s* lp = p;
    double* xbuf = p->hx;
    if (p->part && p->sched.partitions >= 2) {
        lp = p->part->sub;
        int e = part_ensure(p->part, 1);
        if (e) return e;
        xbuf = p->part->xx;
    }
    lp->launch_bflag = p->bflag;
    lp->launch_seg_rows = seg_rows;
    lp->launch_epoch = p->epoch;
    lp->launch_hx = hx_dev;
    int e = plan_solve_f64(lp, p->hb, xbuf, 1, s);
    lp->launch_bflag = nullptr;
    lp->launch_hx = nullptr;
    if (e) return e;
    for (int g = 0; g < nseg; g++) {
        const size_t r0 = (size_t)g * seg_rows, rows = std::min<size_t>(seg_rows, n - r0);
        SPT_CUDA(cudaMemcpyAsync(p->hb + r0, hb + r0, sizeof(double) * rows, cudaMemcpyHostToDevice,
                                 p->copy_stream));
        SPT_CUDA(cudaMemcpyAsync(p->bflag + g, p->epochs + p->epoch, sizeof(int), cudaMemcpyHostToDevice,
                                 p->copy_stream));
    }
    SPT_CUDA(cudaEventRecord(p->ev_copied, p->copy_stream));
    SPT_CUDA(cudaStreamWaitEvent(s, p->ev_copied, 0));  // s's later work also comes after the copies
    return 0;
}

sptrsv_schedule_t default_schedule()
{
    sptrsv_schedule_t s;
    s.variant = SPTRSV_VAR_MULTIROW;
    s.rows_per_warp = 1;
    s.block_warps = 8;
    s.warps_per_sm = 0;
    s.backoff_ns = 0;
    s.ir_max_iters = 2;
    s.band_levels = 64;
    s.cluster_rows = 4096;
    s.partitions = 0;
    return s;
}

// Opt-in to large dynamic shared memory.  The default limit covers static
// plus dynamic shared memory up to 48 KB, so a kernel with static shared
// memory needs the opt-in a little below that.
template <typename K>
cudaError_t allow_smem(K kern, size_t bytes)
{
    if (bytes <= 32 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

int plan_fill_values(sptrsv_plan_s* p, const sp_mat_t* L, cudaStream_t s)
{
    if (p->n == 0) return 0;
    k_plan_fill<<<grid_for((long long)p->n * 32, 256), 256, 0, s>>>(L->ia, L->ja, L->a, p->lev, p->n);
    SPT_CUDA(cudaGetLastError());
    if (p->clu.ptr) {  // rebuild the cluster copy from the new values
        int H = p->clu_H, B = p->clu_B;
        p->clu_H = 0;
        SPT_CUDA(cudaStreamSynchronize(s));
        int e = build_cluster_layout(p, H, B);
        if (e) return e;
    }
    if (p->wave.row) {  // the wave copy
        const int G = p->wave.G;
        SPT_CUDA(cudaStreamSynchronize(s));
        wave_free(p->wave);
        int e = build_wave_layout(p, G, kWaveMaxRows);
        if (e) return e;
    }
    if (p->strip.row) {  // and the strip copy
        const int R = p->strip.R;
        SPT_CUDA(cudaStreamSynchronize(s));
        strip_free(p->strip);
        p->row_strip_R = 0;
        int e = build_strip_layout(p, R);
        if (e) return e;
    }
    if (p->band.rec64) {  // the band records
        SPT_CUDA(cudaStreamSynchronize(s));
        band_free(p->band);
        int e = build_band_layout(p);
        if (e) return e;
    }
    if (p->part) {  // the block system: its warm-ups depend on the values
        const int P = p->part->P;
        SPT_CUDA(cudaStreamSynchronize(s));
        part_free(p);
        int e = build_part(p, P);
        if (!e && p->sched.partitions >= 2) {
            sptrsv_schedule_t inner = p->sched;
            inner.partitions = 0;
            e = sptrsv_plan_set_schedule(p->part->sub, &inner);
        }
        if (e) return e;
    }
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

// One sync-free solve over the plan: FP64 (V = T = double) or FP32.
template <typename V, typename T, typename BT, int OUT>
int plan_launch(sptrsv_plan_s* p, bool f32, const BT* b, T* x, double* x64, int nrhs, cudaStream_t s)
{
    Ctx* c = ctx();
    const sptrsv_schedule_t& sc = p->sched;
    const unsigned long long budget = wait_budget_ns();
    const unsigned backoff = (unsigned)sc.backoff_ns;
    const int n = p->n;
    const int block = 32 * sc.block_warps;
    const int cap = sc.warps_per_sm > 0 ? (sc.warps_per_sm + sc.block_warps - 1) / sc.block_warps : 0;
    auto layout_vals = [&](const SptLayout& l, const V*& val, const V*& dg, const V*& di) {
        if (f32) {
            val = reinterpret_cast<const V*>(l.val32);
            dg = reinterpret_cast<const V*>(l.dg32);
            di = reinterpret_cast<const V*>(l.di32);
        } else {
            val = reinterpret_cast<const V*>(l.val64);
            dg = reinterpret_cast<const V*>(l.dg64);
            di = reinterpret_cast<const V*>(l.di64);
        }
    };
    if (sc.variant == SPTRSV_VAR_BAND && nrhs == 1)
        return band_solve(p, f32, b, sizeof(BT) == 4, x, x64, OUT, s);
    if (sc.variant == SPTRSV_VAR_CLUSTER && nrhs == 1) {
        int e = build_cluster_layout(p, sc.band_levels, sc.cluster_rows);
        if (!e) e = build_cluster_tasks(p, sc.rows_per_warp);
        if (e) return e;
        const V *val, *dg, *di;
        layout_vals(p->clu, val, dg, di);
        PermMat<V> m{p->clu.ptr, p->clu.rowid, p->clu.col, val, dg, di, nullptr};
        auto kern = k_sptrsv_cluster<V, T, BT, OUT>;
        size_t smem = sizeof(T) * (size_t)p->clu_B;
        SPT_CUDA(allow_smem(kern, smem));
        SPT_CUDA(launch_persistent_capped(kern, block, smem, p->nclusters, cap, s, m, (const int*)p->cptr,
                                          (const int*)p->clu_ctask, (const int*)p->clu_tasks, p->nclusters,
                                          32 / sc.rows_per_warp, b, x, x64, c->d_status, budget, backoff));
        return 0;
    }
    if (sc.variant == SPTRSV_VAR_STRIP && nrhs == 1) {
        int e = build_strip_layout(p, sc.rows_per_warp);
        if (e) return e;
        const StripLayout& t = p->strip;
        StripMat<V> m{t.row, t.pe, t.ecol,
                      f32 ? reinterpret_cast<const V*>(t.ev32) : reinterpret_cast<const V*>(t.ev64),
                      f32 ? reinterpret_cast<const V*>(t.lsub32) : reinterpret_cast<const V*>(t.lsub64),
                      f32 ? reinterpret_cast<const V*>(t.di32) : reinterpret_cast<const V*>(t.di64), t.sptr};
        auto kern = k_sptrsv_strip<V, T, BT, OUT>;
        const size_t smem = (size_t)sc.block_warps * t.W * 32 * sizeof(T);
        SPT_CUDA(allow_smem(kern, smem));
        SPT_CUDA(launch_persistent_capped(kern, block, smem, div_up(t.nstrips, sc.block_warps), cap, s, m,
                                          t.nstrips, t.W, b, x, x64, c->d_status, budget, backoff));
        return 0;
    }
    if (sc.variant == SPTRSV_VAR_WAVE && nrhs == 1) {
        int e = build_wave_layout(p, sc.block_warps, kWaveMaxRows);
        if (e) return e;
        const WaveLayout& t = p->wave;
        WaveMat<V> m{{t.row, t.pe, t.ecol,
                      f32 ? reinterpret_cast<const V*>(t.ev32) : reinterpret_cast<const V*>(t.ev64),
                      f32 ? reinterpret_cast<const V*>(t.lsub32) : reinterpret_cast<const V*>(t.lsub64),
                      f32 ? reinterpret_cast<const V*>(t.di32) : reinterpret_cast<const V*>(t.di64), nullptr},
                     t.runc, t.grun, t.grow,
                     // a streamed solve takes the groups in row order, the order b arrives in
                     p->launch_bflag ? nullptr : t.gseq, p->launch_bflag ? t.brow : nullptr,
                     p->launch_bflag ? t.ghx : nullptr};
        auto kern = p->launch_bflag
                        ? (t.maxe <= 2         ? k_sptrsv_wave<V, T, BT, OUT, 2, false, true>
                           : t.maxe <= kStripU ? k_sptrsv_wave<V, T, BT, OUT, kStripU, false, true>
                                               : k_sptrsv_wave<V, T, BT, OUT, kStripU, true, true>)
                        : (t.maxe <= 2         ? k_sptrsv_wave<V, T, BT, OUT, 2, false, false>
                           : t.maxe <= kStripU ? k_sptrsv_wave<V, T, BT, OUT, kStripU, false, false>
                                               : k_sptrsv_wave<V, T, BT, OUT, kStripU, true, false>);
        const size_t smem = (size_t)t.cap * sizeof(T);
        SPT_CUDA(allow_smem(kern, smem));
        SPT_CUDA(launch_persistent_capped(kern, block, smem, t.ngroups, cap, s, m, t.ngroups, b, x, x64, c->d_status,
                                          budget, backoff, p->launch_bflag, p->launch_seg_rows, p->launch_epoch,
                                          p->launch_hx));
        return 0;
    }
    const V *val, *dg, *di;
    layout_vals(p->lev, val, dg, di);
    PermMat<V> m{p->lev.ptr, p->lev.rowid, p->lev.col, val, dg, di,
                 sc.variant == SPTRSV_VAR_SIMPLE ? p->inv : nullptr};
    const int wpb = sc.block_warps;
    if (nrhs > 1) {
        // multi-RHS: level-aligned groups of short rows and pieces of long rows
        PermMat<V> ml = m;
        ml.seq = nullptr;
        int kp = 1, j = 0;
        while (kp < nrhs) kp <<= 1;
        while ((1 << j) < kp) j++;
        // entries per lane per wait round (the table's round size): 16 where levels
        // are wide and the gathers in flight set the pace, 8 where levels are
        // narrow and more resident warps (fewer registers) shorten each hop
        // (measured on B200: Zipf n = 2e6, 16 RHS 3.98 vs 4.53 ms; banded
        // n = 1e5, 16 RHS 4.67 vs 6.53 ms)
        const int U = (long long)p->n >= 1024LL * std::max(1, p->nlevs) ? 16 : 8;
        int e = build_mrhs_tasks(p, kp, U);
        if (e) return e;
        const MrhsTable& t = p->mrhs[j];
        if (t.nsplit) SPT_CUDA(cudaMemsetAsync(t.pcnt, 0, sizeof(int) * (size_t)t.nsplit, s));
        // rows of x a whole number of 16-byte copies wide: gathered through L2 in 16-byte copies
        const bool cg = (nrhs * sizeof(T)) % 16 == 0;
        auto kern = U == 8 ? (cg ? k_sptrsv_mrhs<V, T, BT, OUT, 8, MRHS_CG> : k_sptrsv_mrhs<V, T, BT, OUT, 8, MRHS_CA>)
                           : (cg ? k_sptrsv_mrhs<V, T, BT, OUT, 16, MRHS_CG> : k_sptrsv_mrhs<V, T, BT, OUT, 16, MRHS_CA>);
        // the multi-RHS kernel takes at most 8 warps per block (its register use)
        const int mw = std::min(wpb, 8), mblock = 32 * mw;
        const int mcap = sc.warps_per_sm > 0 ? (sc.warps_per_sm + mw - 1) / mw : 0;
        const size_t smem = (size_t)mw * U * 32 * sizeof(T);
        SPT_CUDA(allow_smem(kern, smem));
        SPT_CUDA(launch_persistent_capped(kern, mblock, smem, div_up(t.ntasks, mw), mcap, s, ml, t.ntasks,
                                          reinterpret_cast<const MrhsTask*>(t.tasks), nrhs, kp, b, x, x64,
                                          reinterpret_cast<T*>(t.pbuf), t.pcnt, c->d_status, budget, backoff));
        return 0;
    }
    if (sc.variant == SPTRSV_VAR_SIMPLE) {
        // natural-order chunks of rows_per_warp rows, solved in sequence by a warp
        auto kern = k_sptrsv_chunk<PermMat<V>, T, BT, OUT>;
        SPT_CUDA(launch_persistent_capped(kern, block, 0, div_up(div_up(n, sc.rows_per_warp), wpb), cap, s, m, n,
                                          sc.rows_per_warp, b, x, x64, c->d_status, budget, backoff));
        return 0;
    }
    auto kern = k_sptrsv<PermMat<V>, T, BT, OUT>;
    if (sc.variant == SPTRSV_VAR_MULTIROW) {
        SPT_CUDA(launch_persistent_capped(kern, block, 0, div_up(p->n_warps, wpb), cap, s, m, n, p->n_warps, 0,
                                          (const int*)p->ibase, (const int*)p->ivect, b, x, x64, c->d_status, budget,
                                          backoff));
    } else {
        // ORDER: level-aligned tasks, rows of one warp never depend on each other
        int j = 0;
        while ((1 << j) < sc.rows_per_warp) j++;
        int e = build_order_tasks(p, sc.rows_per_warp);
        if (e) return e;
        SPT_CUDA(launch_persistent_capped(kern, block, 0, div_up(p->ord_ntasks[j], wpb), cap, s, m, n,
                                          p->ord_ntasks[j], 32 / sc.rows_per_warp, (const int*)p->ord_tasks[j],
                                          (const int*)nullptr, b, x, x64, c->d_status, budget, backoff));
    }
    return 0;
}

int plan_residual(sptrsv_plan_s* p, const double* b, const double* x, float* r32, double* r64, int nrhs,
                  cudaStream_t s)
{
    PermMat<double> m{p->lev.ptr, p->lev.rowid, p->lev.col, p->lev.val64, p->lev.dg64, p->lev.di64, nullptr};
    const int n = p->n;
    if (nrhs > 1) {
        int kp = 1;
        while (kp < nrhs) kp <<= 1;
        long long work = (long long)div_up(n, 32 / kp) * 32;
        if (r32) k_residual_mrhs<float><<<grid_for(work, 256), 256, 0, s>>>(m, n, nrhs, kp, b, x, r32);
        else k_residual_mrhs<double><<<grid_for(work, 256), 256, 0, s>>>(m, n, nrhs, kp, b, x, r64);
    } else {
        int avg = n > 0 ? p->nnz_off / n : 0;
        int L = avg <= 1 ? 1 : avg <= 2 ? 2 : avg <= 4 ? 4 : avg <= 8 ? 8 : avg <= 16 ? 16 : 32;
        long long work = (long long)div_up(n, 32 / L) * 32;
        if (r32) k_residual<float><<<grid_for(work, 256), 256, 0, s>>>(m, n, L, b, x, r32);
        else k_residual<double><<<grid_for(work, 256), 256, 0, s>>>(m, n, L, b, x, r64);
    }
    SPT_CUDA(cudaGetLastError());
    return 0;
}

static bool partitioned(const sptrsv_plan_s* p) { return p->part && p->sched.partitions >= 2; }

int part_gather64(PartPlan* q, const double* src, double* dst, int k, cudaStream_t s);
int part_gather32(PartPlan* q, const float* src, float* dst, int k, cudaStream_t s);
int part_scatter64(PartPlan* q, const double* src, double* dst, int k, cudaStream_t s);
int part_scatter32(PartPlan* q, const float* src, float* out32, double* x64, int mode, int k, cudaStream_t s);

int plan_solve_f64(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s)
{
    if (partitioned(p)) return part_solve_f64(p, b, x, nrhs, s);
    SPT_CUDA(cudaMemsetAsync(x, 0xFF, sizeof(double) * (size_t)p->n * nrhs, s));
    return plan_launch<double, double, double, OUT_X>(p, false, b, x, nullptr, nrhs, s);
}

// Partitioned FP64 solve: b gathered into the block system, solved there,
// each block's real rows scattered into x.
int part_solve_f64(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s)
{
    PartPlan* q = p->part;
    if (q->sub->sched.variant == SPTRSV_VAR_BAND && nrhs == 1)  // records map to this plan's rows
        return band_solve(q->sub, false, b, false, x, nullptr, OUT_X, s);
    int e = part_ensure(q, nrhs);
    if (!e) e = part_gather64(q, b, q->bx, nrhs, s);
    if (!e) e = plan_solve_f64(q->sub, q->bx, q->xx, nrhs, s);
    if (!e) e = part_scatter64(q, q->xx, x, nrhs, s);
    return e;
}

template <typename BT>
int part_solve32(sptrsv_plan_s* p, const BT* rhs, float* out32, double* x64, int out_mode, int nrhs, cudaStream_t s)
{
    PartPlan* q = p->part;
    if (q->sub->sched.variant == SPTRSV_VAR_BAND && nrhs == 1)
        return band_solve(q->sub, true, rhs, sizeof(BT) == 4, out32, x64, out_mode, s);
    int e = part_ensure(q, nrhs);
    if (e) return e;
    const BT* g;
    if constexpr (sizeof(BT) == 8) {
        e = part_gather64(q, rhs, q->bx, nrhs, s);
        g = q->bx;
    } else {
        e = part_gather32(q, rhs, q->bx32, nrhs, s);
        g = q->bx32;
    }
    if (e) return e;
    SPT_CUDA(cudaMemsetAsync(q->xx32, 0xFF, sizeof(float) * (size_t)q->n_ext * nrhs, s));
    e = plan_launch<float, float, BT, OUT_X>(q->sub, true, g, q->xx32, nullptr, nrhs, s);
    if (e) return e;
    return part_scatter32(q, q->xx32, out32, x64, out_mode, nrhs, s);
}
template int part_solve32<double>(sptrsv_plan_s*, const double*, float*, double*, int, int, cudaStream_t);
template int part_solve32<float>(sptrsv_plan_s*, const float*, float*, double*, int, int, cudaStream_t);

// FP32 solve of rhs into out32 (the readiness flags of the unpartitioned
// kernels, so never null there) and, per out_mode, x64 = or += the result.
template <typename BT>
int solve32(sptrsv_plan_s* p, const BT* rhs, float* out32, double* x64, int out_mode, int nrhs, cudaStream_t s)
{
    if (partitioned(p)) return part_solve32<BT>(p, rhs, out32, x64, out_mode, nrhs, s);
    SPT_CUDA(cudaMemsetAsync(out32, 0xFF, sizeof(float) * (size_t)p->n * nrhs, s));
    if (out_mode == OUT_SET64) return plan_launch<float, float, BT, OUT_SET64>(p, true, rhs, out32, x64, nrhs, s);
    if (out_mode == OUT_ADD64) return plan_launch<float, float, BT, OUT_ADD64>(p, true, rhs, out32, x64, nrhs, s);
    return plan_launch<float, float, BT, OUT_X>(p, true, rhs, out32, nullptr, nrhs, s);
}

int plan_solve_ir(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s)
{
    int e = plan_ensure_work(p, nrhs);
    if (e) return e;
    e = solve32<double>(p, b, p->w32a, x, OUT_SET64, nrhs, s);
    if (e) return e;
    for (int it = 0; it < p->sched.ir_max_iters; it++) {
        e = plan_residual(p, b, x, p->w32b, nullptr, nrhs, s);
        if (e) return e;
        e = solve32<float>(p, p->w32b, p->w32a, x, OUT_ADD64, nrhs, s);
        if (e) return e;
    }
    return 0;
}

namespace {

// max |a| into *out as the bit pattern of a non-negative float/double (IEEE
// order of non-negative values is integer order; a NaN reads as the largest)
__global__ void k_absmax32(const float* __restrict__ a, long long m, unsigned* out)
{
    unsigned mx = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        mx = max(mx, __float_as_uint(fabsf(a[i])));
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}
__global__ void k_absmax64(const double* __restrict__ a, long long m, unsigned long long* out)
{
    unsigned long long mx = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        mx = max(mx, (unsigned long long)__double_as_longlong(fabs(a[i])));
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

}  // namespace

// Runs the refinement with up to max_iters steps and returns in *iters the
// fewest steps after which the next correction is below tol relative to x
// (the next correction estimates the remaining error).
int plan_calibrate_ir(sptrsv_plan_s* p, const double* b, double* x, int nrhs, double tol, int max_iters,
                      int* iters, double* last_ratio)
{
    int e = plan_ensure_work(p, nrhs);
    if (e) return e;
    const long long m = (long long)p->n * nrhs;
    unsigned long long* d_n = nullptr;  // [0] |x| (f64 bits), [1] |d| (f32 bits)
    SPT_CUDA(cudaMalloc((void**)&d_n, 2 * sizeof(unsigned long long)));
    cudaStream_t s = 0;
    auto fail = [&](int code) {
        cudaFree(d_n);
        return code;
    };
    e = solve32<double>(p, b, p->w32a, x, OUT_SET64, nrhs, s);
    if (e) return fail(e);
    int need = max_iters;
    double ratio = 0;
    for (int it = 1; it <= max_iters + 1; it++) {
        e = plan_residual(p, b, x, p->w32b, nullptr, nrhs, s);
        if (e) return fail(e);
        e = solve32<float>(p, p->w32b, p->w32a, nullptr, OUT_X, nrhs, s);
        if (e) return fail(e);
        cudaMemsetAsync(d_n, 0, 2 * sizeof(unsigned long long), s);
        k_absmax64<<<grid_for(m, 256), 256, 0, s>>>(x, m, d_n);
        k_absmax32<<<grid_for(m, 256), 256, 0, s>>>(p->w32a, m, reinterpret_cast<unsigned*>(d_n + 1));
        unsigned long long h[2] = {0, 0};
        if (cudaMemcpyAsync(h, d_n, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return fail(cuda_fail(cudaGetLastError(), "calibrate norms"));
        e = sync_status(s);
        if (e) return fail(e);
        double xn = __builtin_bit_cast(double, h[0]);
        double dn = (double)__builtin_bit_cast(float, (unsigned)h[1]);
        ratio = xn > 0 ? dn / xn : dn;
        if (ratio <= tol) {  // x after it-1 steps is within tol
            need = it - 1;
            break;
        }
        if (it == max_iters + 1) break;
        // apply the correction: x += d (the plain solve above wrote d to w32a only)
        e = solve32<float>(p, p->w32b, p->w32a, x, OUT_ADD64, nrhs, s);
        if (e) return fail(e);
    }
    cudaFree(d_n);
    if (iters) *iters = need;
    if (last_ratio) *last_ratio = ratio;
    return 0;
}

int check_schedule(const sptrsv_schedule_t* s)
{
    if (s->variant < 0 || s->variant >= SPTRSV_N_VARIANTS)
        return set_error(SPTRSV_ERR_UNSUPPORTED, "schedule: unknown variant %d", s->variant);
    if (!pow2_lanes(s->rows_per_warp)) return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: rows_per_warp");
    if (s->block_warps != 2 && s->block_warps != 4 && s->block_warps != 8 && s->block_warps != 16)
        return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: block_warps must be 2, 4, 8 or 16");
    if (s->warps_per_sm < 0 || s->warps_per_sm > 64) return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: warps_per_sm");
    if (s->backoff_ns < 0 || s->backoff_ns > 100000) return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: backoff_ns");
    if (s->ir_max_iters < 0 || s->ir_max_iters > 16) return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: ir_max_iters");
    if (s->partitions < 0 || s->partitions > 4096)
        return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: partitions must be in [0, 4096]");
    if (s->band_levels < 1 || s->band_levels > 4096) return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: band_levels");
    if (s->cluster_rows < 32 || s->cluster_rows > 8192)
        return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: cluster_rows must be in [32, 8192]");
    if (s->variant == SPTRSV_VAR_STRIP && strip_smem_bytes(s, 8) > 200 * 1024)
        return set_error(SPTRSV_ERR_INVALID_ARG, "schedule: strip ring does not fit shared memory");
    return 0;
}

}  // namespace sptrsv

using namespace sptrsv;

extern "C" {

void csr_L_solve_simple(sp_mat_t* mat, const VALUE_TYPE* b, VALUE_TYPE* x, int n, int* is_solved)
{
    ::sptrsv::abi_guard_void([&] {
        (void)is_solved;
        solve_reference(mat, nullptr, b, x, n, SIMPLE, 0, 0);
    });
}

void csr_L_solve_order(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b, VALUE_TYPE* x, int n,
                       cudaStream_t stream)
{
    ::sptrsv::abi_guard_void([&] {
        solve_reference(mat, info, b, x, n, ORDER, 32, stream);
    });
}

void csr_L_solve_multirow(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b, VALUE_TYPE* x, int n,
                          cudaStream_t stream)
{
    ::sptrsv::abi_guard_void([&] {
        solve_reference(mat, info, b, x, n, MULTIROW, 0, stream);
    });
}

int sptrsv_solve_order_tile(sp_mat_t* mat, dfr_analysis_info_t* info, const double* b, double* x, int tile,
                            cudaStream_t stream)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!pow2_lanes(tile)) return set_error(SPTRSV_ERR_INVALID_ARG, "order_tile: tile must be 1,2,4,8,16,32");
        return solve_reference(mat, info, b, x, mat ? mat->nr : -1, ORDER, tile, stream);
    });
}

int sptrsv_plan_create(const sp_mat_t* L, const dfr_analysis_info_t* info, sptrsv_plan_t* out)
{
    return ::sptrsv::abi_guard([&]() -> int {
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
        p->sched = default_schedule();
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
        {
            int e = layout_alloc(p->lev, n, p->nnz_off);
            if (e) return fail(e);
        }
        PCHK(dalloc(&p->inv, n));
        PCHK(dalloc(&p->levels, n));
        PCHK(dalloc(&p->ibase, (long long)p->n_warps + 1));
        PCHK(dalloc(&p->ivect, p->n_warps));
        PCHK(dalloc(&d_scr, scan_scratch_ints((long long)n + 1)));
        if (n > 0) {
            k_plan_rows<<<grid_for((long long)n + 1, 256), 256, 0, s>>>(L->ia, info->iorder, n, p->lev.ptr, p->lev.rowid);
            PCHK(cudaGetLastError());
            PCHK(scan_exclusive(p->lev.ptr, p->lev.ptr, (long long)n + 1, d_scr, s));
            int e = plan_fill_values(p, L, s);
            if (e) return fail(e);
            PCHK(cudaMemcpyAsync(p->inv, info->inv_iorder, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s));
            PCHK(cudaMemcpyAsync(p->levels, rec->d_levels, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s));
        }
        PCHK(cudaMemcpyAsync(p->ibase, rec->d_ibase, sizeof(int) * ((size_t)p->n_warps + 1), cudaMemcpyDeviceToDevice, s));
        if (p->n_warps > 0)
            PCHK(cudaMemcpyAsync(p->ivect, rec->d_ivect, sizeof(int) * (size_t)p->n_warps, cudaMemcpyDeviceToDevice, s));
        PCHK(cudaStreamSynchronize(s));
    #undef PCHK
        cudaFree(d_scr);
        *out = p;
        return ok();
    });
}

int sptrsv_plan_destroy(sptrsv_plan_t p)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p) return ok();
        plan_free_arrays(p);
        delete p;
        return ok();
    });
}

int sptrsv_plan_set_schedule(sptrsv_plan_t p, const sptrsv_schedule_t* s)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !s) return set_error(SPTRSV_ERR_INVALID_ARG, "set_schedule: NULL argument");
        int e = check_schedule(s);
        if (e) return e;
        if (s->partitions >= 2) {
            // the variant runs on the block system; if it cannot, the plan keeps
            // the block system its current schedule uses
            PartPlan* prev = p->part;
            e = build_part(p, s->partitions);
            if (e) return e;
            sptrsv_schedule_t inner = *s;
            inner.partitions = 0;
            e = sptrsv_plan_set_schedule(p->part->sub, &inner);
            if (e) {
                if (p->part != prev && p->part_alt == prev) std::swap(p->part, p->part_alt);
                return e;
            }
        } else if (s->variant == SPTRSV_VAR_CLUSTER) {
            e = build_cluster_layout(p, s->band_levels, s->cluster_rows);
            if (!e) e = build_cluster_tasks(p, s->rows_per_warp);
            if (e) return e;
        } else if (s->variant == SPTRSV_VAR_ORDER) {
            e = build_order_tasks(p, s->rows_per_warp);
            if (e) return e;
        } else if (s->variant == SPTRSV_VAR_STRIP) {
            e = build_strip_layout(p, s->rows_per_warp);
            if (e) return e;
        } else if (s->variant == SPTRSV_VAR_WAVE) {
            e = build_wave_layout(p, s->block_warps, kWaveMaxRows);
            if (e) return e;
        } else if (s->variant == SPTRSV_VAR_BAND) {
            e = build_band_layout(p);
            if (e) return e;
        }
        p->sched = *s;
        return ok();
    });
}

int sptrsv_plan_set_stream_segment(sptrsv_plan_t p, int rows)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || rows < 0 || rows % 16 != 0)
            return set_error(SPTRSV_ERR_INVALID_ARG, "set_stream_segment: rows must be 0 or a positive multiple of 16");
        p->seg_rows = rows;
        cudaFree(p->bflag);  // the flag words are sized by the segment count
        p->bflag = nullptr;
        p->nseg = 0;
        return ok();
    });
}

int sptrsv_plan_get_schedule(sptrsv_plan_t p, sptrsv_schedule_t* s)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !s) return set_error(SPTRSV_ERR_INVALID_ARG, "get_schedule: NULL argument");
        *s = p->sched;
        return ok();
    });
}

int sptrsv_plan_update_values(sptrsv_plan_t p, const sp_mat_t* L)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !L || L->nr != p->n || L->nnz - L->nr != p->nnz_off)
            return set_error(SPTRSV_ERR_INVALID_ARG, "update_values: matrix does not match the plan");
        int e = plan_fill_values(p, L, 0);
        if (e) return e;
        SPT_CUDA(cudaStreamSynchronize(0));
        return ok();
    });
}

int sptrsv_solve_f64(sptrsv_plan_t p, const double* b, double* x, int nrhs, cudaStream_t stream)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !b || !x || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "solve_f64: bad arguments");
        if (p->n == 0) return ok();
        int e = plan_solve_f64(p, b, x, nrhs, stream);
        return e ? e : ok();
    });
}

int sptrsv_solve_ir(sptrsv_plan_t p, const double* b, double* x, int nrhs, cudaStream_t stream)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !b || !x || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "solve_ir: bad arguments");
        if (p->n == 0) return ok();
        int e = plan_solve_ir(p, b, x, nrhs, stream);
        return e ? e : ok();
    });
}

int sptrsv_solve_f32(sptrsv_plan_t p, const double* b, float* x32, int nrhs, cudaStream_t stream)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !b || !x32 || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "solve_f32: bad arguments");
        if (p->n == 0) return ok();
        int e = solve32<double>(p, b, x32, nullptr, OUT_X, nrhs, stream);
        return e ? e : ok();
    });
}

int sptrsv_plan_calibrate_ir(sptrsv_plan_t p, const double* b, double* x, int nrhs, double tol, int max_iters,
                             int* iters, double* est)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !b || !x || nrhs < 1 || nrhs > 32 || !(tol > 0) || max_iters < 0 || max_iters > 16)
            return set_error(SPTRSV_ERR_INVALID_ARG, "calibrate_ir: bad arguments");
        if (p->n == 0) {
            if (iters) *iters = 0;
            return ok();
        }
        int need = max_iters;
        double r = 0;
        int e = plan_calibrate_ir(p, b, x, nrhs, tol, max_iters, &need, &r);
        if (e) return e;
        if (r > tol && need >= max_iters) {
            p->sched.ir_max_iters = max_iters;
            if (iters) *iters = need;
            if (est) *est = r;
            return set_error(SPTRSV_ERR_NOT_CONVERGED, "calibrate_ir: correction/x = %.3g after %d steps", r, max_iters);
        }
        p->sched.ir_max_iters = need;
        if (iters) *iters = need;
        if (est) *est = r;
        return ok();
    });
}

int sptrsv_residual_f64(sptrsv_plan_t p, const double* b, const double* x, double* r, int nrhs, cudaStream_t stream)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !b || !x || !r || nrhs < 1 || nrhs > 32) return set_error(SPTRSV_ERR_INVALID_ARG, "residual: bad arguments");
        if (p->n == 0) return ok();
        int e = plan_residual(p, b, x, nullptr, r, nrhs, stream);
        return e ? e : ok();
    });
}

int sptrsv_solve_host(sptrsv_plan_t p, const double* hb, double* hx, int nrhs, int precision, cudaStream_t s)
{
    return ::sptrsv::abi_guard([&]() -> int {
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
        void* hx_dev = nullptr;
        if (nrhs == 1 && precision == 64 && p->sched.variant == SPTRSV_VAR_WAVE && mapped_host(hb) &&
            (hx_dev = mapped_host(hx)) != nullptr) {
            int e = partitioned(p) ? 0 : build_wave_layout(p, p->sched.block_warps, kWaveMaxRows);
            if (!e) e = solve_host_streamed(p, hb, (double*)hx_dev, s);
            if (e) return e;
            e = sync_status(s);
            return e ? e : ok();
        }
        SPT_CUDA(cudaMemcpyAsync(p->hb, hb, bytes, cudaMemcpyHostToDevice, s));
        int e = precision == 32 ? plan_solve_ir(p, p->hb, p->hx, nrhs, s) : plan_solve_f64(p, p->hb, p->hx, nrhs, s);
        if (e) return e;
        SPT_CUDA(cudaMemcpyAsync(hx, p->hx, bytes, cudaMemcpyDeviceToHost, s));
        e = sync_status(s);
        return e ? e : ok();
    });
}

}  // extern "C"
