/*
 * sptrsv_b200.h — C ABI of the B200-native sparse lower-triangular solver.
 *
 * Drop-in boundary for the CSR SpTRSV path of HCL-Fing/SPTRSV.  The first
 * block keeps the reference's types and entry points with the same names,
 * struct layouts, MODE values and parameter orders, wrapped in extern "C" so
 * that a reference caller recompiles unchanged and any FFI (ctypes, cgo, JNI)
 * can bind the symbols by name.  The second block adds new symbols only; no
 * reference symbol changes meaning.
 *
 * Matrix convention (as in the reference): square lower-triangular CSR,
 * 0-based, int32 indices, columns strictly increasing inside a row and the
 * diagonal stored LAST in every row (the reference kernels read
 * val[rowptr[i+1]-1] as the diagonal, solver/solve_csr_simple.cu:45).
 *
 * VALUE_TYPE is fixed to double, the reference's default
 * (Makefile:7, header/common.h:28).  FP32 work happens inside the library.
 *
 * Error behaviour: functions that return int in the reference return 0 on
 * success and a negative SPTRSV_ERR_* code on failure (the reference only
 * printed, header/common.h:163-168).  Functions that return void in the
 * reference record their outcome in a thread-local last error, read with
 * sptrsv_last_error() / sptrsv_last_error_string().  No C++ exception
 * leaves the library: host memory, sizes or threads that cannot be had give
 * SPTRSV_ERR_ALLOC.  No device wait in this library is unbounded: a wait
 * that runs out sets a device status word and returns, and the host reports
 * SPTRSV_ERR_TIMEOUT.
 */
#ifndef SPTRSV_B200_H
#define SPTRSV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifndef VALUE_TYPE
#define VALUE_TYPE double
#endif

/* Same typedef as CUDA's driver_types.h, so both headers can be included. */
struct CUstream_st;
typedef struct CUstream_st* cudaStream_t;

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Reference types (header/dfr_syncfree.h:7-41), same layout and values.      */
/* ------------------------------------------------------------------------- */

/* header/dfr_syncfree.h:7-12 */
typedef enum MODE { SIMPLE = 0, ORDER = 1, MULTIROW = 2, ALL = 3 } MODE;

/* header/dfr_syncfree.h:14-23 — device CSR handle.  ia[nr+1], ja[nnz],
 * a[nnz] are device pointers owned by the library after allocate_memory. */
typedef struct {
    int nr;
    int nc;
    int nnz;
    int* ia;
    int* ja;
    VALUE_TYPE* a;
} sp_mat_t;

/* header/dfr_syncfree.h:25-41 — analysis result.  All pointers are device
 * arrays owned by the library and released by free_device_analysis.
 *   iorder[nr]            rows stably sorted by key 7*(level-1)+bucket
 *   ibase_row[n_warps+1]  first iorder position of each multirow warp
 *   ivect_size_warp[n_warps] lanes per row of each multirow warp (0: diagonal-only rows)
 *   row_ctr[1]            ticket / status word
 * Fields the reference declares but never fills are filled here:
 *   lev_size[nlevs]       rows per level
 *   warp_lev[n_warps]     level (1-based) of each multirow warp
 *   inv_iorder[nr]        position of each row in iorder
 *   lev_ctr               0 */
typedef struct {
    MODE mode;
    int lev_ctr;
    int nlevs;
    int* lev_size;
    int* warp_lev;
    int n_warps;
    int* inv_iorder;
    int* iorder;
    int* ibase_row;
    int* ivect_size_warp;
    int* row_ctr;
} dfr_analysis_info_t;

/* ------------------------------------------------------------------------- */
/* Reference entry points.                                                    */
/* ------------------------------------------------------------------------- */

/* Replaces header/interface.h:6 (defined at interface.cu:9).  Copies a host
 * CSR (n rows, nnz = csrRowPtrL[n]-csrRowPtrL[0]) to the device and fills the
 * caller-allocated *gpu_L.  `mode` is recorded for run_analysis callers that
 * do not set info->mode themselves.  Returns 0, or a negative code when the
 * CSR is not lower triangular with the diagonal last. */
int allocate_memory(int* csrRowPtrL, int* csrColIdxL, VALUE_TYPE* csrValL, int n,
                    sp_mat_t* gpu_L, MODE mode);

/* Replaces header/interface.h:7 (defined at interface.cu:28).  Reads
 * info->mode; returns -1 for SIMPLE (no analysis needed, interface.cu:29),
 * 0 after filling *info, or a negative SPTRSV_ERR_* code. */
int run_analysis(dfr_analysis_info_t* info, sp_mat_t* gpu_L);

/* Replaces header/interface.h:8 (defined at interface.cu:40).  b and x are
 * HOST arrays of n values; x receives the solution of L x = b.  Dispatch as
 * in interface.cu:68-90: SIMPLE when info is NULL, else by info->mode
 * (ORDER, MULTIROW; ALL runs MULTIROW).  Outcome in sptrsv_last_error(). */
void run_solver(sp_mat_t* gpu_L, dfr_analysis_info_t* info, VALUE_TYPE* b, VALUE_TYPE* x, int n);

/* Replaces header/interface.h:9 (defined at interface.cu:97).  Frees every
 * device array of *gpu_L and *info and zeroes the pointers.  The structs
 * themselves stay caller-owned.  Either argument may be NULL. */
void free_device_analysis(sp_mat_t* gpu_L, dfr_analysis_info_t* info);

/* Replaces header/analysis.h:20 (defined at analysis/analysis_csr.cu:272).
 * *info must point to a caller-allocated struct.  Computes levels, nlevs,
 * iorder and, for MULTIROW/ALL, the multirow warp map, bit-exact with the
 * reference.  Outcome in sptrsv_last_error(). */
void multirow_analysis_base_GPU(dfr_analysis_info_t** info, sp_mat_t* gpu_L, MODE mode);

/* Replaces header/solver.h:5 (solver/solve_csr_simple.cu:141).  Sync-free
 * solve in natural row order, no analysis.  b, x are DEVICE arrays.
 * is_solved is accepted for signature compatibility and may be NULL: the
 * kernel uses x itself as the readiness flag.  Runs on the legacy default
 * stream like the reference.  Outcome in sptrsv_last_error() (launch errors
 * only; call sptrsv_sync_status for device-side errors). */
void csr_L_solve_simple(sp_mat_t* mat, const VALUE_TYPE* b, VALUE_TYPE* x, int n, int* is_solved);

/* Replaces header/solver.h:6 (solver/solve_csr_order.cu:171).  Rows in
 * iorder sequence, one warp per row.  b, x are DEVICE arrays; stream-ordered. */
void csr_L_solve_order(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b,
                       VALUE_TYPE* x, int n, cudaStream_t stream);

/* Replaces header/solver.h:7 (solver/solve_csr_multirow.cu:116).  1-32 rows
 * per warp from the analysis warp map.  b, x are DEVICE arrays. */
void csr_L_solve_multirow(sp_mat_t* mat, dfr_analysis_info_t* info, const VALUE_TYPE* b,
                          VALUE_TYPE* x, int n, cudaStream_t stream);

/* ------------------------------------------------------------------------- */
/* Extensions (new symbols; no counterpart changes meaning).                  */
/* ------------------------------------------------------------------------- */

#define SPTRSV_OK                 0
#define SPTRSV_NO_ANALYSIS       -1  /* run_analysis on SIMPLE (interface.cu:29) */
#define SPTRSV_ERR_INVALID_ARG   -2
#define SPTRSV_ERR_INVALID_CSR   -3
#define SPTRSV_ERR_CUDA          -4
#define SPTRSV_ERR_TIMEOUT       -5
#define SPTRSV_ERR_NOT_ANALYSED  -6
#define SPTRSV_ERR_ALLOC         -7
#define SPTRSV_ERR_NOT_CONVERGED -8
#define SPTRSV_ERR_UNSUPPORTED   -9

/* Thread-local outcome of the last call on this host thread. */
int sptrsv_last_error(void);
const char* sptrsv_last_error_string(void);
const char* sptrsv_version(void);

/* Waits for `stream`, then reads and clears the device status word that the
 * kernels of this library set when a bounded wait runs out.  Returns 0 or
 * SPTRSV_ERR_TIMEOUT / SPTRSV_ERR_CUDA. */
int sptrsv_sync_status(cudaStream_t stream);

/* Device-wait budget of every bounded spin in nanoseconds (default 2 s).
 * A wait that exceeds it aborts the kernel with SPTRSV_ERR_TIMEOUT. */
void sptrsv_set_wait_budget_ns(unsigned long long ns);

/* Failure-path self test: one device thread waits on a word that nothing
 * ever writes.  Returns SPTRSV_ERR_TIMEOUT once the bounded wait gives up
 * (after budget_ns); the context stays usable. */
int sptrsv_selftest_bounded_wait(unsigned long long budget_ns);

/* Checks that a HOST CSR is lower triangular with sorted columns and the
 * diagonal last.  Returns 0 or SPTRSV_ERR_INVALID_CSR; *bad_row gets the
 * first offending row (or -1).  Pure host code. */
int sptrsv_check_csr_host(const int* rowptr, const int* colidx, int n, int* bad_row);

/* Copies the 1-based level of every row (the reference's intermediate
 * dfr_analysis_info array, analysis_csr.cu:181) into host_levels[nr]. */
int sptrsv_analysis_levels(const dfr_analysis_info_t* info, int* host_levels);

/* Copies the per-key row counts buckets[7*nlevs] (analysis_csr.cu:336-348)
 * into host_buckets. */
int sptrsv_analysis_buckets(const dfr_analysis_info_t* info, int* host_buckets);

/* Order-coop variant (solver/solve_csr_order.cu:11-77, disabled in the
 * reference by ORDER_COOP 0): iorder sequence, `tile` lanes per row
 * (tile in {1,2,4,8,16,32}).  b, x DEVICE arrays. */
int sptrsv_solve_order_tile(sp_mat_t* mat, dfr_analysis_info_t* info, const double* b,
                            double* x, int tile, cudaStream_t stream);

/* --- Solve plans: the optimised path ------------------------------------- */
/* A plan owns a solve-optimised copy of the matrix built from (gpu_L, info):
 * rows stored in level order, inverse diagonal split out, an FP32 copy of
 * the values, and the chosen schedule.  It does not alias gpu_L->a: after a
 * value change call sptrsv_plan_update_values. */
typedef struct sptrsv_plan_s* sptrsv_plan_t;

/* Solve variants a schedule can pick. */
#define SPTRSV_VAR_SIMPLE    0  /* natural row order, no analysis needed            */
#define SPTRSV_VAR_ORDER     1  /* level order, fixed lanes per row                 */
#define SPTRSV_VAR_MULTIROW  2  /* level order, lanes per row by row length          */
#define SPTRSV_VAR_CLUSTER   3  /* level bands cut into row clusters, one CTA each;  */
                                /* dependencies inside a cluster through shared mem  */
#define SPTRSV_VAR_STRIP     4  /* natural 32-row chunks whose inside dependencies   */
                                /* are all on the previous row, solved by a prefix   */
                                /* scan; rows_per_warp grid lines per warp (1..32),  */
                                /* wavefront order; SPTRSV_ERR_UNSUPPORTED otherwise */
#define SPTRSV_VAR_WAVE      5  /* STRIP's chunks; block_warps grid lines per CTA,   */
                                /* one warp per line, the lines' x in shared memory  */
                                /* (their rows must fit: 25,600 rows in FP64)        */
#define SPTRSV_VAR_BAND      6  /* one warp per independent unit (the matrix, or a  */
                                /* block of a partitioned schedule), level by level, */
                                /* x in a shared-memory ring, no cross-warp waits;   */
                                /* rows of at most 128 off-diagonals, levels of at   */
                                /* most 128 rows on average per unit                 */
#define SPTRSV_N_VARIANTS    7

typedef struct {
    int variant;          /* SPTRSV_VAR_*                                            */
    int rows_per_warp;    /* 1,2,4,8,16,32: lanes per row = 32/rows_per_warp         */
                          /* (MULTIROW takes lanes per row from the analysis map;     */
                          /* STRIP: chunk runs per warp)                              */
    int block_warps;      /* warps per CTA: 2, 4, 8 or 16                             */
    int warps_per_sm;     /* resident warps per SM of the persistent grid (0 = max)   */
    int backoff_ns;       /* nanosleep between polls after 8 failed polls (0 = spin)  */
    int ir_max_iters;     /* FP32+IR: refinement steps after the first FP32 solve     */
    int band_levels;      /* CLUSTER: levels per band (H)                             */
    int cluster_rows;     /* CLUSTER: rows per cluster (B, <= 8192)                   */
    int partitions;       /* 0 or 1: solve L as one system.  P >= 2: cut the rows     */
                          /* into P blocks solved independently by the variant above; */
                          /* block i starts its substitution K_i rows early from a    */
                          /* zero boundary (its warm-up), K_i chosen at plan time so  */
                          /* that a proven bound on the effect of the dropped rows is */
                          /* below 2^-60 relative to max|x|.  Needs a row diagonally  */
                          /* dominant L (|L_ii| >= sum_j |L_ij|) and at least 256     */
                          /* rows per block, else SPTRSV_ERR_UNSUPPORTED.  P <= 4096. */
} sptrsv_schedule_t;

/* Creates a plan for the analysed matrix.  info must come from run_analysis
 * or multirow_analysis_base_GPU on gpu_L (any mode but SIMPLE). */
int sptrsv_plan_create(const sp_mat_t* gpu_L, const dfr_analysis_info_t* info, sptrsv_plan_t* plan);
int sptrsv_plan_destroy(sptrsv_plan_t plan);
int sptrsv_plan_set_schedule(sptrsv_plan_t plan, const sptrsv_schedule_t* s);
int sptrsv_plan_get_schedule(sptrsv_plan_t plan, sptrsv_schedule_t* s);
/* A partitioned plan's blocks (schedule with partitions >= 2): their count,
 * the rows of the block system, the warm-up rows in all, the largest
 * truncation bound (relative to max|x|, <= 2^-60) and, when table is not
 * NULL, 4 ints per block: warm-up start s, first real row a, end e (the
 * next block's a), first row in the block system. */
int sptrsv_plan_partition_info(sptrsv_plan_t plan, int* blocks, int* n_ext, long long* warm_rows,
                               double* bound, int* table);
/* The same blocks computed on the host from a host CSR, without a GPU
 * (table: 4 ints per block as above; *bound the largest truncation bound).
 * SPTRSV_ERR_UNSUPPORTED as for the schedule. */
struct sptrsv_host_csr_s;
int sptrsv_partition_blocks_host(const struct sptrsv_host_csr_s* m, int P, int* table, double* bound);
/* Re-reads gpu_L->a (same pattern) into the plan's value copies. */
int sptrsv_plan_update_values(sptrsv_plan_t plan, const sp_mat_t* gpu_L);

/* Plain FP64 solve of L X = B for nrhs right-hand sides (1..32).  B and X
 * are DEVICE arrays, row-major n x nrhs (value (i,k) at i*nrhs+k). */
int sptrsv_solve_f64(sptrsv_plan_t plan, const double* b, double* x, int nrhs, cudaStream_t stream);

/* FP32 solve with FP64 iterative refinement: x0 = solve32(b); then
 * ir_max_iters times r = b - L x (FP64), d = solve32(r), x += d (FP64).
 * Same layout as sptrsv_solve_f64. */
int sptrsv_solve_ir(sptrsv_plan_t plan, const double* b, double* x, int nrhs, cudaStream_t stream);

/* Picks the number of refinement steps for this plan: runs the FP32 solve
 * and corrections (up to max_iters + 1) on b, and sets ir_max_iters to the
 * fewest steps after which the next correction, relative to x in the
 * inf-norm, is below tol (the next correction estimates the remaining
 * forward error; pass a margin, e.g. tol = 1e-13 for a 1e-12 target).
 * x is a DEVICE scratch/output vector.  *iters and *est (that ratio) may be
 * NULL.  SPTRSV_ERR_NOT_CONVERGED if max_iters steps do not get there. */
int sptrsv_plan_calibrate_ir(sptrsv_plan_t plan, const double* b, double* x, int nrhs, double tol, int max_iters,
                             int* iters, double* est);

/* The inner FP32 solve of sptrsv_solve_ir on its own: x32 (DEVICE, n x nrhs
 * floats) = L^-1 b with FP32 values and accumulation, b read as FP64. */
int sptrsv_solve_f32(sptrsv_plan_t plan, const double* b, float* x32, int nrhs, cudaStream_t stream);

/* Host-buffer convenience of sptrsv_solve_ir / sptrsv_solve_f64 (copies in
 * and out on `stream` through plan-owned device buffers; precision 32 picks
 * FP32+IR, 64 plain FP64).  With a WAVE schedule, precision 64, one
 * right-hand side and both host arrays pinned (cudaHostAlloc or registered),
 * the copies overlap the solve: b goes over in 1 MiB segments on a
 * plan-owned side stream while the kernel runs (it waits for each segment),
 * and the kernel writes x into host_x as groups of rows finish.  Returns
 * after the solve. */
int sptrsv_solve_host(sptrsv_plan_t plan, const double* host_b, double* host_x, int nrhs,
                      int precision, cudaStream_t stream);

/* Rows per segment of b in the streamed host solve (a multiple of 16; 0:
 * the default, an eighth of the rows but at least 131072 = 1 MiB of
 * doubles).  Fewer, larger segments mean fewer copies queued per solve; the
 * kernel starts on the first segment once it has arrived. */
int sptrsv_plan_set_stream_segment(sptrsv_plan_t plan, int rows);

/* FP64 residual r = b - L x on the device (row-major n x nrhs). */
int sptrsv_residual_f64(sptrsv_plan_t plan, const double* b, const double* x, double* r,
                        int nrhs, cudaStream_t stream);

/* --- A solve that allocates nothing --------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory when they solve — code whose device heap is owned by a pool or an
 * arena, or that must not call cudaMalloc after start-up.  The caller passes
 * the device CSR (diagonal last), b and x (DEVICE, n values); no analysis or
 * plan is needed.  FP32 solve in natural-order chunks, then ir_iters
 * (0..16; others give SPTRSV_ERR_INVALID_ARG) refinement steps (FP64
 * residual, FP32 correction, x += d in FP64).  The CSR is not checked on the
 * host: the kernels check every row range and column before they use it, and
 * a CSR that is not lower triangular with the diagonal last gives
 * SPTRSV_ERR_INVALID_CSR.
 * Scratch lives in a fixed file-scope device array (two FP32 vectors of
 * SPTRSV_NOALLOC_MAX_ROWS and a status word, about 8 MiB per GPU, kept until
 * the process exits): n above SPTRSV_NOALLOC_MAX_ROWS is rejected with
 * SPTRSV_ERR_UNSUPPORTED.  CUDA loads a library's device code lazily by
 * default, so the array is reserved on a device when this module is first
 * loaded there — at the first call of this function on that device (or at
 * context creation with CUDA_MODULE_LOADING=EAGER).  That first call also
 * looks up the array's device address.  Make it at start-up, before the
 * pool or arena takes the device heap and before any stream capture.  All
 * calls share the array: calls that overlap on the GPU (other streams or
 * host threads) race, so the caller serialises them.
 * Waits for `stream` and returns 0 or a negative SPTRSV_ERR_* code. */
#define SPTRSV_NOALLOC_MAX_ROWS (1 << 20)
int sptrsv_solve_ir_noalloc(const sp_mat_t* gpu_L, const double* b, double* x, int ir_iters,
                            cudaStream_t stream);

/* --- Batched solves: many systems, one persistent launch ------------------ */
/* nsys independent systems (device CSRs, e.g. from allocate_memory), system s
 * with nrhs[s] right-hand sides (1..32), solved together: one analysis of
 * their block-diagonal union, rows laid out in (level, right-hand-side
 * class) order, one persistent launch per solve, replayable as a CUDA graph.
 * Vectors are packed: system s owns the row-major n_s x nrhs[s] block that
 * starts at element offsets[s] (sptrsv_batch_info).  The batch keeps its own
 * copy of the matrices. */
typedef struct sptrsv_batch_s* sptrsv_batch_t;
int sptrsv_batch_create(int nsys, const sp_mat_t* mats, const int* nrhs, sptrsv_batch_t* out);
int sptrsv_batch_destroy(sptrsv_batch_t batch);
/* offsets[nsys+1] (may be NULL), total rows, levels of the union, packed length. */
int sptrsv_batch_info(sptrsv_batch_t batch, long long* offsets, int* n_total, int* nlevs, long long* vec_len);
/* mode 0: level-ordered tasks over the union;
 * mode 1: each warp takes 32 consecutive rows of one system and solves them
 *         in sequence, waiting once per chunk for the chunks it reads;
 * mode 2 (default): hybrid - every system with n_s / nlevs_s below the sequential
 *         width (sptrsv_batch_set_seq_width) is solved by one warp in
 *         natural order without waiting, the others by level-ordered tasks,
 *         all in the same launch.
 * block_warps 2..16 (2..8 in mode 1).  Rebuilds the level layout when the
 * set of sequential systems changes. */
int sptrsv_batch_set_schedule(sptrsv_batch_t batch, int mode, int block_warps, int warps_per_sm,
                              int backoff_ns, int ir_iters);
/* Width threshold of mode 2 (default 16): a system is sequential when
 * n_s / nlevs_s < width and all its dependencies reach back at most
 * 1024 / kp rows (kp = power of two >= its right-hand-side count), or 1024
 * rows for a system with more than 8 right-hand sides or of at least 16384
 * rows with several (solved one right-hand side per warp); 0 makes no system
 * sequential, >= 1e9 makes every system sequential. */
int sptrsv_batch_set_seq_width(sptrsv_batch_t batch, double width);
/* Systems solved sequentially, warps they occupy, rows left to the level tasks. */
int sptrsv_batch_seq_systems(sptrsv_batch_t batch, int* nseq, int* nseq_warps, int* n_level_rows);
/* Partitioned batch: every system of at least 2 * block_rows rows whose
 * rows are all diagonally dominant is cut into about n_s / block_rows blocks
 * solved independently after a warm-up (see sptrsv_schedule_t.partitions:
 * each block starts early from a zero boundary, far enough that a proven
 * bound on the dropped rows' effect is below 2^-60 relative to max|x|); the
 * blocks and the other systems are solved as one batch of their own, b
 * gathered into it and x scattered back inside every solve (and graph).
 * block_rows: 0 (plain batch) or >= 256.  Keeps the schedule. */
int sptrsv_batch_set_partition(sptrsv_batch_t batch, int block_rows);
/* Systems cut into blocks, systems of the inner batch, warm-up rows in all,
 * the largest truncation bound. */
int sptrsv_batch_partition_info(sptrsv_batch_t batch, int* systems_cut, int* inner_systems, long long* warm_rows,
                                double* bound);
/* b, x: DEVICE packed vectors; precision 64 plain FP64, 32 FP32 + FP64 refinement. */
int sptrsv_batch_solve(sptrsv_batch_t batch, const double* b, double* x, int precision, cudaStream_t stream);
/* Same solve captured once as a CUDA graph for these (b, x, precision) and
 * replayed on `stream`; a different (b, x, precision) captures again. */
int sptrsv_batch_solve_graph(sptrsv_batch_t batch, const double* b, double* x, int precision,
                             cudaStream_t stream);

/* --- Schedule selection: features, autotuner, learned selector ------------ */

/* 12 cheap features of an analysed matrix: log2 n, log2 nnz, nnz/n,
 * log2 nlevs, log2 mean level width, log2 max level width, the 25/50/90/99%
 * quantiles of off-diagonals per row, log2(1 + max off-diagonals per row),
 * fraction of diagonal-only rows. */
int sptrsv_features(const sp_mat_t* gpu_L, const dfr_analysis_info_t* info, float* out12);

/* 24 schedule classes = 4 variants x 6 parameter presets (class = 6*variant + j). */
#define SPTRSV_N_CLASSES 24
int sptrsv_schedule_from_class(int cls, sptrsv_schedule_t* out);

/* Exhaustive autotuner: times every class on this plan (median of `reps`
 * solves after one warm-up, L2 flushed between solves; precision 64 = plain
 * FP64, 32 = FP32 + FP64 refinement), leaves the fastest set on the plan.
 * b, x are DEVICE arrays (n x nrhs); times_ms[24] (may be NULL) receives each
 * class's median, NaN for a class that could not run. */
int sptrsv_autotune(sptrsv_plan_t plan, const double* b, double* x, int nrhs, int precision, int reps,
                    float* times_ms, int* best_class);

/* The learned selector: an MLP 12 -> 64 -> 64 -> 24 (ReLU) that predicts each
 * class's log2(time / best time) from the features; trained and evaluated by
 * the library's own CUDA kernels.  Parameters are 6552 floats, weights
 * row-major [in][out]: W1[12][64] b1[64] W2[64][64] b2[64] W3[64][24] b3[24]. */
typedef struct sptrsv_mlp_s* sptrsv_mlp_t;
#define SPTRSV_MLP_NPARAMS 6552
int sptrsv_mlp_create(uint64_t seed, sptrsv_mlp_t* out);
int sptrsv_mlp_destroy(sptrsv_mlp_t mlp);
int sptrsv_mlp_get_params(sptrsv_mlp_t mlp, float* host_params);
int sptrsv_mlp_set_params(sptrsv_mlp_t mlp, const float* host_params);
/* Inputs are normalised as (x - mean) / std before the first layer. */
int sptrsv_mlp_set_normalization(sptrsv_mlp_t mlp, const float* mean12, const float* std12);
int sptrsv_mlp_get_normalization(sptrsv_mlp_t mlp, float* mean12, float* std12);
/* Y[B x 24] for raw features X[B x 12] (host arrays). */
int sptrsv_mlp_forward_host(sptrsv_mlp_t mlp, const float* X, int B, float* Y);
/* Masked MSE loss and its gradient (6552 floats) at the current parameters:
 * L = sum M (Y - T)^2 / max(1, sum M). */
int sptrsv_mlp_gradient_host(sptrsv_mlp_t mlp, const float* X, const float* T, const float* M, int B,
                             float* grad, float* loss);
/* Minibatch Adam on the device over N rows; loss_curve[epochs] may be NULL. */
int sptrsv_mlp_train_host(sptrsv_mlp_t mlp, const float* X, const float* T, const float* M, int N, int epochs,
                          int batch, float lr, uint64_t seed, float* loss_curve);
/* argmin of the predicted relative times. */
int sptrsv_mlp_predict_class(sptrsv_mlp_t mlp, const float* features12, int* cls);
/* Features -> MLP -> schedule, set on the plan. */
int sptrsv_plan_select_schedule(sptrsv_plan_t plan, sptrsv_mlp_t mlp, const sp_mat_t* gpu_L,
                                const dfr_analysis_info_t* info, int* cls_out);

/* --- Synthetic inputs (host code) ---------------------------------------- */
/* The reference reads SuiteSparse .mtx files (main.cu:66-246); none ship with
 * it.  These seeded generators make the benchmark matrices: square
 * lower-triangular CSR, sorted columns, diagonal last.  Arrays are malloc'd;
 * release them with sptrsv_host_csr_free. */
typedef struct sptrsv_host_csr_s {
    int n;
    int nnz;
    int* rowptr;
    int* colidx;
    double* val;
} sptrsv_host_csr_t;

/* Row i: k ~ U{off_min..off_max} (capped by the window) distinct columns
 * uniform in [max(0,i-bandwidth), i-1]; off-diagonals U(-1,1), diagonal
 * 1 + sum|offdiag|. */
int sptrsv_gen_banded(int n, int bandwidth, int off_min, int off_max, uint64_t seed, sptrsv_host_csr_t* out);
/* Strict lower triangle plus diagonal of the 5-point Laplacian on an nx x ny
 * grid (row-major): neighbours -1 + U(-0.1,0.1), diagonal 4. */
int sptrsv_gen_grid2d(int nx, int ny, uint64_t seed, sptrsv_host_csr_t* out);
/* Same for the 7-point Laplacian on nx x ny x nz, diagonal 6. */
int sptrsv_gen_grid3d(int nx, int ny, int nz, uint64_t seed, sptrsv_host_csr_t* out);
/* Off-diagonal count min(Z-1, max_off, i), Z ~ Zipf(s) on {1,2,...};
 * columns distinct, uniform over all preceding rows; diagonally dominant. */
int sptrsv_gen_zipf(int n, double s, int max_off, uint64_t seed, sptrsv_host_csr_t* out);
/* Block diagonal with dense lower-triangular blocks; diagonally dominant. */
int sptrsv_gen_blockdiag(int n, int block, uint64_t seed, sptrsv_host_csr_t* out);
void sptrsv_host_csr_free(sptrsv_host_csr_t* m);
/* MatrixMarket coordinate file (real/integer/pattern; general, symmetric or
 * skew-symmetric) -> the lower triangle as CSR with sorted columns and the
 * diagonal last in every row (added where the file has none), the extraction
 * of the reference's driver (main.cu:66-246).  unit_values = 1 sets every
 * value to 1.0 as the reference does (main.cu:228,236); 0 keeps the file's
 * values (a missing diagonal gets 1.0).  Duplicates are summed. */
int sptrsv_read_mtx_lower(const char* path, int unit_values, sptrsv_host_csr_t* out);
/* dist 0: ones, 1: U(-1,1), 2: N(0,1). */
int sptrsv_gen_vector(long long m, int dist, uint64_t seed, double* out);
/* y = L x on the host, row-major nrhs. */
int sptrsv_host_spmv(const sptrsv_host_csr_t* m, const double* x, double* y, int nrhs);

#ifdef __cplusplus
}
#endif

#endif /* SPTRSV_B200_H */
