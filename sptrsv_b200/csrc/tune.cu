// tune.cu — the schedule classes, the exhaustive autotuner and the MLP's
// schedule prediction.
//
// 24 classes = 4 groups x 6 parameter presets.  The natural-order group holds
// SIMPLE with 1 and 32 rows per task, STRIP with one grid line per warp and
// WAVE with 4, 8 and 16 grid lines per CTA (STRIP and WAVE apply only to
// matrices with their chunk structure, WAVE only where a line group fits
// shared memory; elsewhere those classes fail to set and are skipped).  For
// ORDER the preset is rows per warp (1..32, i.e. 32..1 lanes per row — the
// reference's six tile sizes, analysis_csr.cu:84-102).  MULTIROW takes lanes per row from the analysis
// map, so its presets vary the polling back-off and the number of resident
// warps.  CLUSTER presets vary band height, cluster size and lanes per row.
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
    if (!s || cls < 0 || cls >= SPTRSV_N_CLASSES) return set_error(SPTRSV_ERR_INVALID_ARG, "schedule_from_class: bad class");
    static const int rpw[6] = {1, 2, 4, 8, 16, 32};
    // natural-order group: SIMPLE with 1 and 32 rows per task; between them
    // STRIP with one grid line per warp and WAVE with 4, 8, 16 lines per CTA
    static const int nat_v[6] = {SPTRSV_VAR_SIMPLE, SPTRSV_VAR_STRIP, SPTRSV_VAR_WAVE, SPTRSV_VAR_WAVE,
                                 SPTRSV_VAR_WAVE, SPTRSV_VAR_SIMPLE};
    static const int nat_bw[6] = {8, 2, 4, 8, 16, 8};
    // MULTIROW presets: block warps, back-off ns, resident warps per SM
    static const int mr[6][3] = {{8, 0, 0}, {8, 200, 0}, {8, 1000, 0}, {4, 0, 16}, {8, 200, 32}, {16, 0, 0}};
    // CLUSTER presets: band levels, cluster rows, rows per warp, block warps
    // (from sweeps of H = 16..4096, B = 1024..8192 on banded and grid matrices:
    // wide bands with 16 rows per task and 16-warp blocks lead)
    static const int cl[6][4] = {{64, 4096, 16, 8},    {128, 4096, 16, 16}, {256, 2048, 16, 16},
                                 {256, 4096, 16, 16},  {512, 8192, 16, 16}, {4096, 2048, 16, 8}};
    const int v = cls / 6, j = cls % 6;
    s->variant = v;
    s->rows_per_warp = 1;
    s->block_warps = 8;
    s->warps_per_sm = 0;
    s->backoff_ns = 0;
    s->ir_max_iters = 2;
    s->band_levels = 64;
    s->cluster_rows = 4096;
    s->partitions = 0;
    if (v == SPTRSV_VAR_SIMPLE && nat_v[j] != SPTRSV_VAR_SIMPLE) {
        s->variant = nat_v[j];
        s->rows_per_warp = 1;
        s->block_warps = nat_bw[j];
    } else if (v == SPTRSV_VAR_SIMPLE || v == SPTRSV_VAR_ORDER) {
        s->rows_per_warp = rpw[j];
    } else if (v == SPTRSV_VAR_MULTIROW) {
        s->block_warps = mr[j][0];
        s->backoff_ns = mr[j][1];
        s->warps_per_sm = mr[j][2];
    } else {
        s->band_levels = cl[j][0];
        s->cluster_rows = cl[j][1];
        s->rows_per_warp = cl[j][2];
        s->block_warps = cl[j][3];
    }
    return ok();
}

int sptrsv_autotune(sptrsv_plan_t p, const double* b, double* x, int nrhs, int precision, int reps, float* times_ms,
                    int* best_class)
{
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
}

int sptrsv_mlp_forward_host(sptrsv_mlp_t M, const float* X, int B, float* Y);

int sptrsv_mlp_predict_class(sptrsv_mlp_t M, const float* features12, int* cls)
{
    if (!M || !features12 || !cls) return set_error(SPTRSV_ERR_INVALID_ARG, "mlp_predict_class: NULL");
    float y[SPTRSV_N_CLASSES];
    int e = sptrsv_mlp_forward_host(M, features12, 1, y);
    if (e) return e;
    int best = 0;
    for (int c = 1; c < SPTRSV_N_CLASSES; c++)
        if (y[c] < y[best]) best = c;
    *cls = best;
    return ok();
}

int sptrsv_plan_select_schedule(sptrsv_plan_t p, sptrsv_mlp_t M, const sp_mat_t* L, const dfr_analysis_info_t* info,
                                int* cls_out)
{
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
}

}  // extern "C"
