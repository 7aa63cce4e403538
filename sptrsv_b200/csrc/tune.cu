// tune.cu — the schedule classes, the exhaustive autotuner and the MLP's
// schedule prediction.
//
// 24 classes = 4 groups x 6 parameter presets (one table, below).  The
// natural-order group holds SIMPLE, STRIP and WAVE, whole and over 16 blocks
// with warm-ups (STRIP and WAVE apply only to matrices with their chunk
// structure, WAVE only where a line group fits shared memory; elsewhere those
// classes fail to set and are skipped).  For ORDER the preset is rows per
// warp (1..32, i.e. 32..1 lanes per row — the reference's six tile sizes,
// analysis_csr.cu:84-102).  MULTIROW takes lanes per row from the analysis
// map; its presets vary the polling back-off and resident warps, and cut the
// rows into 16 or 128 blocks.  The last group holds CLUSTER and BAND, whole
// and over blocks.  Partitioned classes use 16 or 128 blocks only, so an
// autotune builds at most two block systems (a plan keeps the last two).
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "internal.h"
#include "plan.h"

namespace sptrsv {
int plan_solve_f64(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s);
int plan_solve_ir(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s);
}  // namespace sptrsv

using namespace sptrsv;

extern "C" {

int sptrsv_schedule_from_class(int cls, sptrsv_schedule_t* s)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!s || cls < 0 || cls >= SPTRSV_N_CLASSES) return set_error(SPTRSV_ERR_INVALID_ARG, "schedule_from_class: bad class");
        // preset: {variant, rows_per_warp, block_warps, warps_per_sm, backoff_ns, band_levels, cluster_rows, partitions}
        static const int T[SPTRSV_N_CLASSES][8] = {
            // natural order / wavefront: SIMPLE 32 rows per task, STRIP one line per warp, WAVE 8 and 4 lines
            // per CTA, and WAVE over 16 blocks with warm-ups (4 and 8 lines per CTA)
            {SPTRSV_VAR_SIMPLE, 32, 8, 0, 0, 64, 4096, 0},   {SPTRSV_VAR_STRIP, 1, 2, 0, 0, 64, 4096, 0},
            {SPTRSV_VAR_WAVE, 1, 8, 0, 0, 64, 4096, 0},      {SPTRSV_VAR_WAVE, 1, 4, 0, 0, 64, 4096, 0},
            {SPTRSV_VAR_WAVE, 1, 4, 0, 0, 64, 4096, 16},     {SPTRSV_VAR_WAVE, 1, 8, 0, 0, 64, 4096, 16},
            // ORDER: the reference's six tile sizes (analysis_csr.cu:84-102), 32..1 lanes per row
            {SPTRSV_VAR_ORDER, 1, 8, 0, 0, 64, 4096, 0},     {SPTRSV_VAR_ORDER, 2, 8, 0, 0, 64, 4096, 0},
            {SPTRSV_VAR_ORDER, 4, 8, 0, 0, 64, 4096, 0},     {SPTRSV_VAR_ORDER, 8, 8, 0, 0, 64, 4096, 0},
            {SPTRSV_VAR_ORDER, 16, 8, 0, 0, 64, 4096, 0},    {SPTRSV_VAR_ORDER, 32, 8, 0, 0, 64, 4096, 0},
            // MULTIROW over the reference's lane map: its own setting (class 12), back-off, fewer resident
            // warps, 16-warp blocks, and over 16 and 128 blocks with warm-ups
            {SPTRSV_VAR_MULTIROW, 1, 8, 0, 0, 64, 4096, 0},  {SPTRSV_VAR_MULTIROW, 1, 8, 0, 200, 64, 4096, 0},
            {SPTRSV_VAR_MULTIROW, 1, 4, 16, 0, 64, 4096, 0}, {SPTRSV_VAR_MULTIROW, 1, 16, 0, 0, 64, 4096, 0},
            {SPTRSV_VAR_MULTIROW, 1, 8, 0, 0, 64, 4096, 16}, {SPTRSV_VAR_MULTIROW, 1, 8, 0, 0, 64, 4096, 128},
            // CLUSTER (bands of H levels cut into clusters of B rows) and BAND (one warp per unit), whole and
            // over blocks with warm-ups
            {SPTRSV_VAR_CLUSTER, 16, 16, 0, 0, 256, 2048, 0}, {SPTRSV_VAR_CLUSTER, 16, 8, 0, 0, 4096, 2048, 0},
            {SPTRSV_VAR_BAND, 1, 8, 0, 0, 64, 4096, 0},       {SPTRSV_VAR_CLUSTER, 16, 16, 0, 0, 256, 2048, 16},
            {SPTRSV_VAR_BAND, 1, 8, 0, 0, 64, 4096, 16},      {SPTRSV_VAR_BAND, 1, 8, 0, 0, 64, 4096, 128},
        };
        const int* t = T[cls];
        s->variant = t[0];
        s->rows_per_warp = t[1];
        s->block_warps = t[2];
        s->warps_per_sm = t[3];
        s->backoff_ns = t[4];
        s->ir_max_iters = 2;
        s->band_levels = t[5];
        s->cluster_rows = t[6];
        s->partitions = t[7];
        return ok();
    });
}

int sptrsv_autotune(sptrsv_plan_t p, const double* b, double* x, int nrhs, int precision, int reps, float* times_ms,
                    int* best_class)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !b || !x || nrhs < 1 || nrhs > 32 || (precision != 32 && precision != 64) || reps < 1)
            return set_error(SPTRSV_ERR_INVALID_ARG, "autotune: bad arguments");
        if (p->n == 0) return ok();
        const size_t flush_bytes = 256u << 20;
        void* flush = nullptr;
        SPT_CUDA(cudaMalloc(&flush, flush_bytes));
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        const sptrsv_schedule_t saved = p->sched;
        float best_t = std::numeric_limits<float>::infinity();
        int best = -1;
        for (int cls = 0; cls < SPTRSV_N_CLASSES; cls++) {
            sptrsv_schedule_t s;
            sptrsv_schedule_from_class(cls, &s);
            s.ir_max_iters = saved.ir_max_iters;
            float med = std::numeric_limits<float>::quiet_NaN();
            if (sptrsv_plan_set_schedule(p, &s) == 0) {
                std::vector<float> ts;
                bool bad = false;
                for (int r = 0; r <= reps && !bad; r++) {  // first run is a warm-up
                    cudaMemsetAsync(flush, r & 0xff, flush_bytes, 0);
                    cudaEventRecord(e0, 0);
                    int e = precision == 64 ? plan_solve_f64(p, b, x, nrhs, 0) : plan_solve_ir(p, b, x, nrhs, 0);
                    cudaEventRecord(e1, 0);
                    if (e || sync_status(0)) {
                        bad = true;
                        break;
                    }
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (r > 0) ts.push_back(ms);
                }
                if (!bad) {
                    std::sort(ts.begin(), ts.end());
                    med = ts[ts.size() / 2];
                    if (med < best_t) {
                        best_t = med;
                        best = cls;
                    }
                }
            }
            if (times_ms) times_ms[cls] = med;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(flush);
        if (best < 0) {
            p->sched = saved;
            return set_error(SPTRSV_ERR_CUDA, "autotune: no schedule ran");
        }
        sptrsv_schedule_t s;
        sptrsv_schedule_from_class(best, &s);
        s.ir_max_iters = saved.ir_max_iters;
        sptrsv_plan_set_schedule(p, &s);
        if (best_class) *best_class = best;
        return ok();
    });
}

int sptrsv_mlp_forward_host(sptrsv_mlp_t M, const float* X, int B, float* Y);

int sptrsv_mlp_predict_class(sptrsv_mlp_t M, const float* features12, int* cls)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!M || !features12 || !cls) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_predict_class: NULL");
        float y[SPTRSV_N_CLASSES];
        int e = sptrsv_mlp_forward_host(M, features12, 1, y);
        if (e) return e;
        int best = 0;
        for (int c = 1; c < SPTRSV_N_CLASSES; c++)
            if (y[c] < y[best]) best = c;
        *cls = best;
        return ok();
    });
}

int sptrsv_plan_select_schedule(sptrsv_plan_t p, sptrsv_mlp_t M, const sp_mat_t* L, const dfr_analysis_info_t* info,
                                int* cls_out)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p || !M || !L || !info) return set_error(SPTRSV_ERR_INVALID_ARG, "select_schedule: NULL");
        float f[12];
        int e = sptrsv_features(L, info, f);
        if (e) return e;
        // classes in order of predicted time; the first one that applies to
        // this matrix (STRIP and WAVE classes need its chunk structure) is set
        float out[SPTRSV_N_CLASSES];
        e = sptrsv_mlp_forward_host(M, f, 1, out);
        if (e) return e;
        int order[SPTRSV_N_CLASSES];
        for (int k = 0; k < SPTRSV_N_CLASSES; k++) order[k] = k;
        std::stable_sort(order, order + SPTRSV_N_CLASSES, [&](int a, int b) { return out[a] < out[b]; });
        for (int k = 0; k < SPTRSV_N_CLASSES; k++) {
            sptrsv_schedule_t s;
            sptrsv_schedule_from_class(order[k], &s);
            s.ir_max_iters = p->sched.ir_max_iters;
            if (sptrsv_plan_set_schedule(p, &s) == 0) {
                if (cls_out) *cls_out = order[k];
                return ok();
            }
        }
        return set_error(SPTRSV_ERR_UNSUPPORTED, "select_schedule: no class applies");
    });
}

}  // extern "C"
