// plan.h — the solve plan: solve-optimised copies of L.
//
// A layout stores the rows in a schedule order so that the rows a warp (or
// CTA) works on are contiguous (n rows, m = nnz - n off-diagonal entries):
//   ptr[n+1]    int32   off-diagonal offsets per position
//   rowid[n]    int32   original row of each position (b, x are indexed by it)
//   col[m]      int32   off-diagonal column (original index; in the cluster
//                       layout ~local for a column inside the same cluster)
//   val64[m]    f64     off-diagonal values
//   val32[m]    f32     the same values rounded to FP32
//   dg64[n], dg32[n]    diagonal per position
//   di64[n], di32[n]    its reciprocal (the reference's piv = 1/diag)
// The level layout (iorder sequence) is always built; it serves SIMPLE
// (through inv[n], natural row -> position), ORDER, MULTIROW (with the
// analysis warp map ibase/ivect) and the FP64 residual.  The cluster layout
// is built when a CLUSTER schedule is set, for its (band_levels,
// cluster_rows), with cptr[nclusters+1] giving each cluster's positions.
// Work buffers: w32a/w32b (n x nrhs f32) for the FP32 solves and residuals,
// hb/hx (n x nrhs f64) staging for the host-buffer entry point.
#pragma once

#include <vector>

#include "sptrsv_b200.h"

struct SptLayout {
    int* ptr = nullptr;
    int* rowid = nullptr;
    int* col = nullptr;
    double* val64 = nullptr;
    float* val32 = nullptr;
    double* dg64 = nullptr;
    float* dg32 = nullptr;
    double* di64 = nullptr;  // 1 / diagonal, rounded once in f64
    float* di32 = nullptr;   // 1.0f / (float)diagonal
};

// STRIP schedule (built on demand, see strip.cu).  Arrays are in processing
// order: slot P * 32 + j is row j of the chunk at position P (strips
// contiguous, positions of a strip in its wavefront order).
struct StripLayout {
    int* row = nullptr;        // [npos*32] natural row of the slot, -1 past the last row
    int* pe = nullptr;         // [npos*32+1] first entry of the slot (entries before its chunk)
    int* ecol = nullptr;       // column, or ~ring slot for a chunk this warp solved recently
    double* ev64 = nullptr;
    float* ev32 = nullptr;
    double* lsub64 = nullptr;  // [npos*32] L(i, i-1) when row i-1 is in the same chunk, else 0
    float* lsub32 = nullptr;
    double* di64 = nullptr;    // [npos*32] 1 / diagonal
    float* di32 = nullptr;
    int* sptr = nullptr;       // [nstrips+1] first position of each strip
    int nstrips = 0, R = 0, W = 0;
};

// WAVE schedule (built on demand, see strip.cu): the strip chunks in natural
// order (slot = chunk * 32 + lane); G consecutive runs (grid lines) form a
// group solved by one CTA, one warp per line, with the group's x values in
// shared memory.
struct WaveLayout {
    int* row = nullptr;        // [nch*32] natural row of the slot, -1 past the chunk's last row
    int* pe = nullptr;         // [nch*32+1] first entry of the slot
    int* ecol = nullptr;       // column, or ~(column - first row of the group) inside the group
    double* ev64 = nullptr;
    float* ev32 = nullptr;
    double* lsub64 = nullptr;
    float* lsub32 = nullptr;
    double* di64 = nullptr;
    float* di32 = nullptr;
    int* runc = nullptr;       // [nruns+1] first chunk of each run
    int* grun = nullptr;       // [ngroups+1] first run of each group
    int* grow = nullptr;       // [ngroups+1] first row of each group
    int* gseq = nullptr;       // [ngroups] processing order of the groups (null: natural order)
    int* brow = nullptr;       // block systems only: [nch*32] outer row whose b a slot takes
    int* ghx = nullptr;        // block systems only: [ngroups*2] outer row of a group's first row,
                               // its first row that is not a warm-up row
    int ngroups = 0, G = 0, cap = 0;  // cap: most rows in one group
    int maxe = 0;                      // most entries of one slot
};

// Multi-RHS task table for kp = 1 << j lanes per row (built on demand, see
// mrhs.cu): 8 ints per task (MrhsTask), level-aligned, each level's pieces of
// long rows first, then its groups of short rows.
struct MrhsTable {
    int* tasks = nullptr;   // [ntasks * 8]
    int ntasks = 0;
    int npslots = 0;        // partial-sum slots (pieces of rows cut in more than one piece)
    int nsplit = 0;         // rows cut in more than one piece (one counter each)
    void* pbuf = nullptr;   // [npslots * kp] partial sums (f64; f32 solves use the front half)
    int* pcnt = nullptr;    // [nsplit] piece counters, cleared before each launch
    int U = 0;              // elements per lane per wait round the table was cut for
};

// BAND schedule (built on demand, see band.cu): per unit (the whole matrix,
// or each block of a block system) the steps of its levels as fixed-size
// records, FP64 and FP32 copies.
constexpr int kBandU = 4;  // entries per lane per step
struct BandLayout {
    int U = 0, R = 0;          // entries per lane per step; ring slots (slot R is a constant 0)
    int nunits = 0, nsteps = 0;
    int* ustep = nullptr;      // [nunits+1] first step of each unit
    unsigned char* rec64 = nullptr;  // [nsteps * rb64]
    unsigned char* rec32 = nullptr;  // [nsteps * rb32]
    int rb64 = 0, rb32 = 0;
    int* bidx = nullptr;       // [nsteps * 32] row whose b a lane's row takes (-1: none)
};

// Partitioned solve (built on demand, see part.cu): the rows are cut into P
// blocks; block i covers the real rows [a_i, e_i) and starts its substitution
// at s_i <= a_i from a zero boundary.  The blocks, with every entry that
// points before their start dropped, form one block-diagonal system of
// n_ext rows (block i at rows base_i ...) that a plan of its own (sub)
// solves with any variant; b is gathered into it and x scattered out of it.
struct PartPlan {
    int P = 0;
    int n_ext = 0;
    long long nnz_ext = 0;
    long long warm_rows = 0;      // sum of a_i - s_i
    double bound = 0;             // largest truncation bound of a block (relative to max|x|)
    int reach = 0;                // most rows between an entry's column and its row
    std::vector<int> tab;         // [P * 4]: s_i, a_i, e_i, base_i
    int* d_tab = nullptr;
    sp_mat_t ext{};               // device CSR of the block system
    dfr_analysis_info_t info{};   // its analysis
    struct sptrsv_plan_s* sub = nullptr;
    double* bx = nullptr;         // [n_ext * nrhs] gathered right-hand sides
    double* xx = nullptr;         // [n_ext * nrhs] block-system solution
    float* bx32 = nullptr;        // FP32 gathered residuals
    float* xx32 = nullptr;        // FP32 block-system solutions
    int cap_rhs = 0;
};

struct sptrsv_plan_s {
    int device = -1;
    int n = 0, nnz_off = 0, nlevs = 0, n_warps = 0;
    SptLayout lev;               // level order
    int* inv = nullptr;          // natural row -> level-layout position
    int* levels = nullptr;       // 1-based level per row
    int* ibase = nullptr;        // multirow map
    int* ivect = nullptr;
    int* ord_tasks[6] = {};      // level-aligned tasks over the level layout, R = 1 << j rows
    int ord_ntasks[6] = {};
    SptLayout clu;               // cluster order (built on demand)
    int* cptr = nullptr;
    int* clu_key = nullptr;      // per position: cluster * H + local level
    int nclusters = 0, clu_H = 0, clu_B = 0;
    int* clu_tasks = nullptr;    // (cluster, level)-aligned tasks
    int* clu_ctask = nullptr;    // first task of each cluster [nclusters+1]
    int clu_ntasks = 0, clu_R = 0;
    MrhsTable mrhs[6];           // multi-RHS tables per kp = 1 << j (built on demand)
    StripLayout strip;           // STRIP layout (built on demand)
    int row_strip_R = 0;         // R the strip layout was built for (0: none)
    WaveLayout wave;             // WAVE layout (built on demand)
    // streamed host solves (WAVE, FP64): b copied in segments on a side
    // stream while the kernel runs, one flag word per segment
    int* bflag = nullptr;        // [nseg] epoch of the last copy of each segment
    int nseg = 0;
    int* epochs = nullptr;       // pinned host table: epochs[e] = e, the flag values' source
    int epoch = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_copied = nullptr;
    const int* launch_bflag = nullptr;  // set only during a streamed launch
    int launch_epoch = 0;
    int launch_seg_rows = 0;
    int seg_rows = 0;            // rows per copied segment of b (0: the default, 1 MiB of doubles)
    double* launch_hx = nullptr;
    float* w32a = nullptr;
    float* w32b = nullptr;
    int cap_rhs = 0;
    double* hb = nullptr;
    double* hx = nullptr;
    int cap_host = 0;
    sptrsv_schedule_t sched{};
    PartPlan* part = nullptr;    // partitioned solve (sched.partitions >= 2)
    PartPlan* part_alt = nullptr;  // the previous block system, kept for a switch back
    // set on a block system's plan: the first row of every block (WAVE
    // groups never span two blocks, and the blocks' groups are interleaved)
    std::vector<int> blk_starts;
    // set on a block system's plan: the outer plan's block table (s, a, e,
    // base per block), so BAND records can read b and write x in the outer
    // plan's rows directly
    std::vector<int> part_tab;
    BandLayout band;             // BAND layout (built on demand)
};

namespace sptrsv {
void layout_free(SptLayout& l);
int layout_alloc(SptLayout& l, int n, int m);
// Builds (or rebuilds) p->clu for (H, B) from the level layout.
int build_cluster_layout(sptrsv_plan_s* p, int H, int B);
// Level-aligned task tables with R rows per task (cached per R).
int build_order_tasks(sptrsv_plan_s* p, int R);
int build_cluster_tasks(sptrsv_plan_s* p, int R);
// Builds (or keeps) p->strip for R runs per strip; SPTRSV_ERR_UNSUPPORTED
// when the matrix does not have the chunk structure.
int build_strip_layout(sptrsv_plan_s* p, int R);
void strip_free(StripLayout& t);
// Builds (or keeps) p->wave for G lines per CTA; SPTRSV_ERR_UNSUPPORTED when
// the matrix does not have the chunk structure or a group's rows do not fit
// max_rows.
int build_wave_layout(sptrsv_plan_s* p, int G, int max_rows);
void wave_free(WaveLayout& w);
// Builds (or keeps) the multi-RHS task table for kp lanes per row.
int build_mrhs_tasks(sptrsv_plan_s* p, int kp, int U);
void mrhs_free(MrhsTable& t);
// Builds (or keeps) p->band; SPTRSV_ERR_UNSUPPORTED when a row is too long,
// levels are too wide for one warp, or the ring would not fit.
int build_band_layout(sptrsv_plan_s* p);
void band_free(BandLayout& t);
// One BAND solve of the plan (see band.cu): b FP64 or FP32 (b_f32); FP64
// (x double) or FP32 (x float, may be null; x64 per out_mode) arithmetic.
int band_solve(sptrsv_plan_s* p, bool f32, const void* b, bool b_f32, void* x, double* x64, int out_mode,
               cudaStream_t s);
// Builds (or keeps) p->part for P blocks; SPTRSV_ERR_UNSUPPORTED when L is
// not row diagonally dominant or too small to cut.
int build_part(sptrsv_plan_s* p, int P);
void part_free(sptrsv_plan_s* p);
// Block-system vectors for nrhs right-hand sides (kept, grown on demand).
int part_ensure(PartPlan* q, int k);
// Partitioned solves (p->sched.partitions >= 2, p->part built).
int part_solve_f64(sptrsv_plan_s* p, const double* b, double* x, int nrhs, cudaStream_t s);
// FP32 solve of the block system for rhs (FP64 or FP32, n x nrhs): out32 =
// L^-1 rhs, and x64 = out32 (OUT_SET64), x64 += out32 (OUT_ADD64) or
// nothing (OUT_X).
template <typename BT>
int part_solve32(sptrsv_plan_s* p, const BT* rhs, float* out32, double* x64, int out_mode, int nrhs,
                 cudaStream_t s);
}  // namespace sptrsv
