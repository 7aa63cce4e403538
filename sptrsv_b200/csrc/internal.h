// internal.h — host-side internals shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <exception>
#include <mutex>
#include <new>
#include <stdexcept>
#include <system_error>
#include <unordered_map>

#include "common.cuh"
#include "sptrsv_b200.h"

namespace sptrsv {

// ---- errors --------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
inline int ok() { return set_error(SPTRSV_OK, "ok"); }
int cuda_fail(cudaError_t e, const char* where);

#define SPT_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return ::sptrsv::cuda_fail(e_, #call);         \
    } while (0)

// Every entry point of the C ABI runs its body through one of these, so no
// C++ exception crosses the ABI: host memory, sizes or threads that cannot be
// had (std::bad_alloc, std::length_error, std::system_error) become
// SPTRSV_ERR_ALLOC, anything else SPTRSV_ERR_INVALID_ARG, with the message in
// the thread's last error.  The void entry points (the reference's solver
// and run_solver signatures) report through the last error only.
template <class F>
int abi_guard(F&& f) noexcept
{
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return set_error(SPTRSV_ERR_ALLOC, "out of host memory");
    } catch (const std::length_error& e) {
        return set_error(SPTRSV_ERR_ALLOC, "host allocation too large: %s", e.what());
    } catch (const std::system_error& e) {
        return set_error(SPTRSV_ERR_ALLOC, "host resources: %s", e.what());
    } catch (const std::exception& e) {
        return set_error(SPTRSV_ERR_INVALID_ARG, "%s", e.what());
    } catch (...) {
        return set_error(SPTRSV_ERR_INVALID_ARG, "unknown exception");
    }
}
template <class F>
void abi_guard_void(F&& f) noexcept
{
    abi_guard([&]() -> int {
        f();
        return 0;
    });
}

// ---- per-device context -------------------------------------------------
struct Ctx {
    int device = -1;
    int num_sms = 0;
    DevStatus* d_status = nullptr;  // one status block per device
};
Ctx* ctx();  // context of the current device (created on first use)
unsigned long long wait_budget_ns();

// Reads and clears the device status after synchronising `stream`.
int sync_status(cudaStream_t stream);

// ---- launches ------------------------------------------------------------
// Grid for a persistent kernel: every block co-resident (occupancy x SMs),
// capped by `max_blocks` and by `cap_per_sm` blocks per SM (0: no cap).
// Launched cooperatively so the co-residency that the static round-robin
// schedule relies on is guaranteed by the driver.
template <typename... KArgs>
cudaError_t persistent_grid(void (*kern)(KArgs...), int block, size_t smem, long long max_blocks, int cap_per_sm,
                            long long* grid_out)
{
    static std::mutex mu;
    static std::unordered_map<long long, int> occ;  // (kernel, block, smem, device) -> blocks per SM
    Ctx* c = ctx();
    long long key = (long long)(uintptr_t)kern ^ ((long long)block << 40) ^ ((long long)smem << 20) ^ c->device;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = occ.find(key);
        if (it == occ.end()) {
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, smem);
            if (e != cudaSuccess) return e;
            occ[key] = per_sm;
        } else {
            per_sm = it->second;
        }
    }
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    if (cap_per_sm > 0 && per_sm > cap_per_sm) per_sm = cap_per_sm;
    long long grid = (long long)per_sm * c->num_sms;
    if (max_blocks < grid) grid = max_blocks;
    if (grid < 1) grid = 1;
    *grid_out = grid;
    return cudaSuccess;
}

// Cooperative launch of a persistent kernel: blocks per SM from the
// occupancy calculator (optionally capped), at most max_blocks blocks, all
// co-resident.
template <typename... KArgs, typename... Args>
cudaError_t launch_persistent_capped(void (*kern)(KArgs...), int block, size_t smem, long long max_blocks,
                                     int cap_per_sm, cudaStream_t s, Args... args)
{
    long long grid = 0;
    cudaError_t e = persistent_grid(kern, block, smem, max_blocks, cap_per_sm, &grid);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
    if (e != cudaSuccess) cudaGetLastError();  // reported here; not left for the next check to find
    return e;
}

template <typename... KArgs, typename... Args>
cudaError_t launch_persistent(void (*kern)(KArgs...), int block, size_t smem, long long max_blocks, cudaStream_t s,
                              Args... args)
{
    return launch_persistent_capped(kern, block, smem, max_blocks, 0, s, args...);
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Grid for a plain grid-stride kernel: enough blocks for `work` threads,
// at most 16 per SM.
int grid_for(long long work, int block);

template <typename T>
cudaError_t dalloc(T** p, long long count)
{
    if (count < 1) count = 1;
    return cudaMalloc((void**)p, sizeof(T) * (size_t)count);
}

// ---- device primitives (util.cu) ----------------------------------------
// Exclusive scan of m ints; in and out may alias.  Needs scratch of
// scan_scratch_ints(m) ints.
long long scan_scratch_ints(long long m);
cudaError_t scan_exclusive(const int* in, int* out, long long m, int* scratch, cudaStream_t s);
// Stable LSD radix sort of (key, val) pairs, keys in [0, max_key].  Uses the
// *_tmp arrays as ping-pong buffers; the sorted result always ends in
// keys/vals.  Scratch: radix_scratch_ints(n) ints.
long long radix_scratch_ints(long long n);
cudaError_t radix_sort_pairs(int* keys, int* vals, int* keys_tmp, int* vals_tmp, long long n, int max_key,
                             int* scratch, cudaStream_t s);
// Segment-aligned task table.  key[p] (p < n) is non-decreasing, in [0, K);
// a segment is a run of equal keys.  Tasks are runs of at most R positions
// inside one segment, so rows of one task never depend on each other when a
// segment is (part of) a level.  R <= 0 takes R = 32 >> (key % 6) per
// segment (keys that carry a lane class in their low base-6 digit).
// *tbase gets ntasks+1 entries (allocated here; tbase[ntasks] = n).
// Returns 0 or an error code.
int build_task_table(const int* key, int n, int K, int R, int** tbase, int* ntasks, cudaStream_t s);

// ---- analysis record -------------------------------------------------------
// Arrays the reference computes internally but does not put in
// dfr_analysis_info_t; kept per analysis, keyed by the info->row_ctr device
// pointer, which is unique per analysis and survives struct copies.
struct AnalysisRec {
    int device = -1;
    int n = 0, nnz = 0, nlevs = 0, n_warps = 0;
    int* d_levels = nullptr;   // [n] 1-based level per row
    int* d_counts = nullptr;   // [7*nlevs+1] rows per key
    int* d_ibase = nullptr;    // [n_warps+1] multirow map (always built)
    int* d_ivect = nullptr;    // [n_warps]
    int* d_wlev = nullptr;     // [n_warps]
    bool map_in_info = false;  // map arrays are also referenced by the info struct
    int* tile_tasks[6] = {};   // level-aligned iorder tasks for 32>>j lanes per row
    int tile_ntasks[6] = {};
};
void register_analysis(const int* key, AnalysisRec* rec);

// Task order for the level kernel: task t covers the cnt[t] <= 32 rows from
// r0[t]; null keeps consecutive 32-row chunks in natural order.
struct LevelTasks {
    const int* r0;
    const int* cnt;
    long long n;
};
// The analysis behind run_analysis / multirow_analysis_base_GPU.
int run_analysis_impl(dfr_analysis_info_t* info, const sp_mat_t* L, MODE mode, const LevelTasks* tasks = nullptr);
AnalysisRec* find_analysis(const int* key);
AnalysisRec* unregister_analysis(const int* key);

}  // namespace sptrsv
