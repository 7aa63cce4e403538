// common.cuh — device helpers shared by the analysis and solve kernels.
//
// Readiness protocol (the reference's NaN-sentinel scheme,
// solver/solve_csr_order.cu:180 and :258-260, with explicit memory order):
// before a solve the output vector is filled with all-ones bits; a row's
// value is its own readiness flag.  Writers store the finished value with a
// relaxed gpu-scope store, readers poll with relaxed gpu-scope loads (L2,
// no L1 allocation).  The value is the only datum passed, and a naturally
// aligned 32/64-bit access is single-copy atomic, so relaxed order suffices
// and no fence sits on the dependency path.  A computed value whose bits
// equal the sentinel (a negative NaN with all mantissa bits set) is replaced
// by the canonical quiet NaN so that readers never wait on a finished row.
//
// Every wait is bounded: it polls a device status word and a %globaltimer
// deadline; on expiry it records SPTRSV_ERR_TIMEOUT and the row, and every
// other waiting warp leaves at its next poll of the status word.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sptrsv_b200.h"

namespace sptrsv {

constexpr int kWarp = 32;

// Device status block: [0] error code (0 = ok), [1] first offending row.
struct DevStatus {
    int code;
    int row;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double ld_relaxed(const double* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return __longlong_as_double((long long)v);
}
__device__ __forceinline__ float ld_relaxed(const float* p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return __uint_as_float(v);
}
__device__ __forceinline__ int ld_relaxed(const int* p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int atom_add_acq_rel(int* p, int v)
{
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_relaxed(double* p, double v)
{
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"((unsigned long long)__double_as_longlong(v))
                 : "memory");
}
__device__ __forceinline__ void st_relaxed(float* p, float v)
{
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(__float_as_uint(v)) : "memory");
}
__device__ __forceinline__ void st_relaxed(int* p, int v)
{
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Sentinel tests: the fill pattern is all-ones bits (memset 0xFF).  For
// doubles the reference tests the high word only (solve_csr_order.cu:260).
__device__ __forceinline__ bool is_pending(double v) { return __double2hiint(v) == (int)0xFFFFFFFF; }
__device__ __forceinline__ bool is_pending(float v) { return __float_as_uint(v) == 0xFFFFFFFFu; }
// Levels are >= 1 once written; the level array is zero-filled.
__device__ __forceinline__ bool is_pending(int v) { return v == 0; }

__device__ __forceinline__ double publishable(double v)
{
    return __double2hiint(v) == (int)0xFFFFFFFF ? __longlong_as_double(0x7FF8000000000000LL) : v;
}
__device__ __forceinline__ float publishable(float v)
{
    return __float_as_uint(v) == 0xFFFFFFFFu ? __uint_as_float(0x7FC00000u) : v;
}

__device__ __forceinline__ void report(DevStatus* st, int code, int row)
{
    if (atomicCAS(&st->code, 0, code) == 0) st->row = row;
}

// Spin until *p is no longer the sentinel.  Returns false if the wait ran out
// or another warp reported an error (the caller then leaves the kernel).
// After 8 failed polls the loop sleeps `backoff_ns` between polls (0: spin),
// which keeps far-ahead waiters from flooding L2 with polls.
template <typename T>
__device__ __forceinline__ bool wait_ready(const T* p, T& out, DevStatus* st, unsigned long long budget_ns, int row,
                                           unsigned backoff_ns = 0)
{
    T v = ld_relaxed(p);
    if (!is_pending(v)) {
        out = v;
        return true;
    }
    unsigned long long t0 = global_ns();
    unsigned it = 0;
    while (true) {
        v = ld_relaxed(p);
        if (!is_pending(v)) {
            out = v;
            return true;
        }
        ++it;
        if (backoff_ns && it > 8) __nanosleep(backoff_ns);
        if ((it & 63u) == 0) {
            if (ld_relaxed(&st->code) != 0) return false;
            if (global_ns() - t0 > budget_ns) {
                report(st, SPTRSV_ERR_TIMEOUT, row);
                return false;
            }
        }
    }
}

// The same wait on a shared-memory slot written by another warp of the CTA.
template <typename T>
__device__ __forceinline__ bool wait_ready_smem(const volatile T* p, T& out, DevStatus* st,
                                                unsigned long long budget_ns, int row)
{
    T v = *p;
    if (!is_pending(v)) {
        out = v;
        return true;
    }
    unsigned long long t0 = global_ns();
    unsigned it = 0;
    while (true) {
        v = *p;
        if (!is_pending(v)) {
            out = v;
            return true;
        }
        if ((++it & 255u) == 0) {
            if (ld_relaxed(&st->code) != 0) return false;
            if (global_ns() - t0 > budget_ns) {
                report(st, SPTRSV_ERR_TIMEOUT, row);
                return false;
            }
        }
    }
}

// Warp-convergent wait: every lane with `pending` set polls its slot (shared
// memory when SMEM and c < 0, else x[c] in global memory) and the whole warp
// loops until all of them are ready.  No lane spins while another lane of
// its warp sits at a sync point: that divergent pattern lets a warp make
// progress only when the scheduler switches paths, which measured several
// microseconds per dependency on B200.  Must be called by all 32 lanes.
// Returns false (warp-uniform) if the wait ran out or another warp reported
// an error.
template <bool SMEM, typename T>
__device__ __forceinline__ bool warp_wait(bool pending, int c, const T* x, const volatile T* xs, T& xv,
                                          DevStatus* st, unsigned long long budget, unsigned backoff, int row)
{
    unsigned long long t0 = 0;
    unsigned it = 0;
    while (true) {
        if (pending) {
            xv = (SMEM && c < 0) ? xs[~c] : ld_relaxed(x + c);
            pending = is_pending(xv);
        }
        if (!__any_sync(0xffffffffu, pending)) return true;
        ++it;
        if (backoff && it > 8) __nanosleep(backoff);
        if ((it & 63u) == 0) {
            int stop = 0;
            if ((threadIdx.x & 31) == 0) {
                unsigned long long now = global_ns();
                if (t0 == 0) t0 = now;
                if (ld_relaxed(&st->code) != 0) stop = 1;
                else if (now - t0 > budget) {
                    report(st, SPTRSV_ERR_TIMEOUT, row);
                    stop = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, stop, 0)) return false;
        }
    }
}

// warp_wait for U values per lane at once: the first nh (per lane) of
// x[c[0..U)] are loaded back to back, so their latencies overlap, and the warp
// spins (convergently, with the same budget and abort rules) only while some
// lane still holds a pending one.  With SMEM, c < 0 reads xs[~c].  Must be
// called by all 32 lanes; returns false (warp-uniform) on timeout or abort.
template <bool SMEM, int U, typename T, typename I>
__device__ __forceinline__ bool warp_wait_n(int nh, const I (&c)[U], const T* x, const volatile T* xs, T (&xv)[U],
                                            DevStatus* st, unsigned long long budget, unsigned backoff, int row)
{
    unsigned pend = 0;
#pragma unroll
    for (int u = 0; u < U; u++) {
        if (u < nh) {
            xv[u] = (SMEM && c[u] < 0) ? xs[~c[u]] : ld_relaxed(x + c[u]);
            if (is_pending(xv[u])) pend |= 1u << u;
        }
    }
    if (!__any_sync(0xffffffffu, pend != 0)) return true;
    unsigned long long t0 = 0;
    unsigned it = 0;
    while (true) {
        ++it;
        if (backoff && it > 8) __nanosleep(backoff);
        if ((it & 63u) == 0) {
            int stop = 0;
            if ((threadIdx.x & 31) == 0) {
                unsigned long long now = global_ns();
                if (t0 == 0) t0 = now;
                if (ld_relaxed(&st->code) != 0) stop = 1;
                else if (now - t0 > budget) {
                    report(st, SPTRSV_ERR_TIMEOUT, row);
                    stop = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, stop, 0)) return false;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if ((pend >> u) & 1u) {
                xv[u] = (SMEM && c[u] < 0) ? xs[~c[u]] : ld_relaxed(x + c[u]);
                if (!is_pending(xv[u])) pend &= ~(1u << u);
            }
        }
        if (!__any_sync(0xffffffffu, pend != 0)) return true;
    }
}

// Warp-convergent bounded wait until *flag == want for every lane with
// need set (acquire: later loads see what was written before the flag).
// Same contract as warp_wait.
__device__ __forceinline__ bool warp_wait_flag(bool need, const int* flag, int want, DevStatus* st,
                                               unsigned long long budget, int row)
{
    unsigned long long t0 = 0;
    unsigned it = 0;
    bool pending = need && ld_acquire(flag) != want;
    while (__any_sync(0xffffffffu, pending)) {
        ++it;
        if ((it & 63u) == 0) {
            int stop = 0;
            if ((threadIdx.x & 31) == 0) {
                unsigned long long now = global_ns();
                if (t0 == 0) t0 = now;
                if (ld_relaxed(&st->code) != 0) stop = 1;
                else if (now - t0 > budget) {
                    report(st, SPTRSV_ERR_TIMEOUT, row);
                    stop = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, stop, 0)) return false;
        }
        if (pending) pending = ld_acquire(flag) != want;
    }
    return true;
}

template <typename T>
__device__ __forceinline__ T sentinel_value();
template <>
__device__ __forceinline__ double sentinel_value<double>()
{
    return __longlong_as_double(-1LL);
}
template <>
__device__ __forceinline__ float sentinel_value<float>()
{
    return __uint_as_float(0xFFFFFFFFu);
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

}  // namespace sptrsv
