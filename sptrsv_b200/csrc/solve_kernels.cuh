// solve_kernels.cuh — sync-free lower-triangular solve kernels.
//
// Arithmetic per row, as in the reference kernels
// (solver/solve_csr_order.cu:238-278, solve_csr_multirow.cu:63-113):
//   left_sum = b_r - sum_j L_rj * x_j   (lanes hold strided partial sums,
//                                         then a segmented shuffle reduction)
//   x_r      = left_sum * (1 / L_rr)
// and, for rows with no off-diagonal in the multirow map, x_r = b_r / L_rr
// (solve_csr_multirow.cu:56-59).
//
// Scheduling: a persistent, co-resident grid; task t goes to warp t mod W
// (cluster c to CTA c mod G) and every warp walks its tasks in increasing
// order.  Tasks are laid out in a topological order, so the lowest
// unfinished task never waits on anything unfinished: no deadlock and no
// ticket atomics (the reference takes one global atomicAdd per warp,
// solve_csr_order.cu:224).
//
// Matrix access goes through a layout policy:
//   NatMat   — the caller's CSR (ia, ja, a) plus an optional row sequence
//              (iorder), exactly the data the reference kernels read;
//   PermMat  — the plan's copy: rows stored in schedule order, off-diagonal
//              entries only (diagonal split out), FP64 or FP32 values.  In
//              the cluster layout a column c < 0 names the row at local
//              position ~c of the same cluster (its value is in shared memory).
#pragma once

#include "common.cuh"

namespace sptrsv {

struct RowRef {
    int r;  // original row index (b and x are indexed by it)
    int s;  // first off-diagonal entry
    int e;  // one past the last off-diagonal entry
    int d;  // where the diagonal lives (entry index or row position)
};

struct NatMat {
    const int* __restrict__ rowptr;
    const int* __restrict__ col;
    const double* __restrict__ val;
    const int* __restrict__ seq;  // null: natural order
    typedef double V;
    __device__ __forceinline__ RowRef row(int pos) const
    {
        RowRef q;
        q.r = seq ? __ldg(seq + pos) : pos;
        q.s = __ldg(rowptr + q.r);
        q.e = __ldg(rowptr + q.r + 1) - 1;
        q.d = q.e;
        return q;
    }
    __device__ __forceinline__ double diag(const RowRef& q) const { return __ldg(val + q.d); }
    __device__ __forceinline__ int c(int p) const { return __ldg(col + p); }
    __device__ __forceinline__ double v(int p) const { return __ldg(val + p); }
};

template <typename VT>
struct PermMat {
    const int* __restrict__ ptr;    // [n+1] off-diagonal offsets per position
    const int* __restrict__ rowid;  // [n] original row of each position
    const int* __restrict__ col;    // off-diagonal columns (original indices)
    const VT* __restrict__ val;     // off-diagonal values
    const VT* __restrict__ dg;      // [n] diagonal per position
    const int* __restrict__ seq;    // null: layout order; else natural -> position
    typedef VT V;
    __device__ __forceinline__ RowRef row(int pos) const
    {
        RowRef q;
        int k = seq ? __ldg(seq + pos) : pos;
        q.r = __ldg(rowid + k);
        q.s = __ldg(ptr + k);
        q.e = __ldg(ptr + k + 1);
        q.d = k;
        return q;
    }
    __device__ __forceinline__ VT diag(const RowRef& q) const { return __ldg(dg + q.d); }
    __device__ __forceinline__ int c(int p) const { return __ldg(col + p); }
    __device__ __forceinline__ VT v(int p) const { return __ldg(val + p); }
};

// Output modes: write x only; also x64 = x; also x64 += x.
enum { OUT_X = 0, OUT_SET64 = 1, OUT_ADD64 = 2 };

template <typename T, int OUT>
__device__ __forceinline__ void publish(T* x, double* x64, size_t i, T v)
{
    st_relaxed(x + i, publishable(v));
    if (OUT == OUT_SET64) x64[i] = (double)v;
    if (OUT == OUT_ADD64) x64[i] += (double)v;
}

__device__ __forceinline__ unsigned segment_mask(int L, int seg)
{
    return L == 32 ? 0xffffffffu : (((1u << L) - 1u) << (seg * L));
}

// Single right-hand side.  Task t: `lanes` lanes per row, 32/lanes rows.
// No table: task t covers positions [t*R, t*R+R) with fixed lanes.
// Table: task t covers [task_base[t], task_base[t+1]) with task_lanes[t]
// lanes per row (the multirow map; 0: diagonal-only rows, one lane each) or,
// when task_lanes is null, with fixed lanes (level-aligned tasks).
template <class M, typename T, typename BT, int OUT>
__global__ void __launch_bounds__(512) k_sptrsv(M m, int npos, int ntasks, int fixed_lanes,
                                                const int* __restrict__ task_base,
                                                const int* __restrict__ task_lanes, const BT* __restrict__ b, T* x,
                                                double* x64, DevStatus* st, unsigned long long budget,
                                                unsigned backoff)
{
    const int lane = threadIdx.x & 31;
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    for (int t = gw; t < ntasks; t += nw) {
        int L, base, cnt;
        if (task_base) {
            base = __ldg(task_base + t);
            cnt = __ldg(task_base + t + 1) - base;
            L = task_lanes ? __ldg(task_lanes + t) : fixed_lanes;
        } else {
            L = fixed_lanes;
            base = t * (32 / L);
            cnt = min(32 / L, npos - base);
        }
        if (L == 0) {  // diagonal-only rows: x = b / diag
            if (lane < cnt) {
                RowRef q = m.row(base + lane);
                T v = (T)b[q.r] / (T)m.diag(q);
                publish<T, OUT>(x, x64, q.r, v);
            }
            continue;
        }
        // Rows of one task may depend on each other (fixed lanes over level or
        // natural order), so each row's lanes reduce and publish on their own
        // (segment mask); the warp converges only after every row published.
        const int seg = lane / L, sl = lane & (L - 1);
        const unsigned smask = segment_mask(L, seg);
        const bool act = seg < cnt;
        T acc = 0;
        bool fail = false;
        RowRef q;
        T piv = 0;
        if (act) {
            q = m.row(base + seg);
            piv = (T)1 / (T)m.diag(q);
            if (sl == 0) acc = (T)b[q.r];
            for (int p = q.s + sl; p < q.e; p += L) {
                int c = m.c(p);
                T v = (T)m.v(p);
                T xv;
                if (!wait_ready(x + c, xv, st, budget, q.r, backoff)) {
                    fail = true;
                    break;
                }
                acc -= v * xv;
            }
        }
        for (int o = L >> 1; o >= 1; o >>= 1) acc += __shfl_down_sync(smask, acc, o, L);
        const bool seg_fail = __any_sync(smask, fail);
        if (act && sl == 0 && !seg_fail) publish<T, OUT>(x, x64, q.r, acc * piv);
        if (__any_sync(0xffffffffu, seg_fail)) return;
    }
}

// Cluster schedule: CTA g processes clusters g, g+G, ...; cluster c holds the
// positions [cptr[c], cptr[c+1]) in level order and the level-aligned tasks
// [ctask[c], ctask[c+1]) (task t: positions [tbase[t], tbase[t+1])).  The
// CTA's warps walk the cluster's tasks round-robin; a dependency inside the
// cluster is read from shared memory (the slot is the flag, filled with the
// sentinel when the cluster starts), one outside it from x in global memory.
template <typename V, typename T, typename BT, int OUT>
__global__ void __launch_bounds__(512) k_sptrsv_cluster(PermMat<V> m, const int* __restrict__ cptr,
                                                        const int* __restrict__ ctask, const int* __restrict__ tbase,
                                                        int nclusters, int L, const BT* __restrict__ b, T* x,
                                                        double* x64, DevStatus* st, unsigned long long budget,
                                                        unsigned backoff)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    volatile T* xs = reinterpret_cast<volatile T*>(smem_raw);
    __shared__ int abort_flag;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nwb = blockDim.x >> 5;
    const int seg = lane / L, sl = lane & (L - 1);
    const unsigned smask = segment_mask(L, seg);
    for (int c = blockIdx.x; c < nclusters; c += gridDim.x) {
        const int cs = __ldg(cptr + c), cn = __ldg(cptr + c + 1) - cs;
        for (int i = threadIdx.x; i < cn; i += blockDim.x) xs[i] = sentinel_value<T>();
        if (threadIdx.x == 0) abort_flag = 0;
        __syncthreads();
        const int t0 = __ldg(ctask + c), t1 = __ldg(ctask + c + 1);
        for (int t = t0 + wib; t < t1; t += nwb) {
            const int tb = __ldg(tbase + t), tcnt = __ldg(tbase + t + 1) - tb;
            const int loc = tb - cs + seg;
            const bool act = seg < tcnt;
            T acc = 0;
            bool fail = false;
            RowRef q;
            T piv = 0;
            if (act) {
                q = m.row(cs + loc);
                piv = (T)1 / (T)m.diag(q);
                if (sl == 0) acc = (T)b[q.r];
                for (int p = q.s + sl; p < q.e; p += L) {
                    int cc = m.c(p);
                    T v = (T)m.v(p);
                    T xv;
                    bool okw = cc < 0 ? wait_ready_smem(xs + (~cc), xv, st, budget, q.r)
                                      : wait_ready(x + cc, xv, st, budget, q.r, backoff);
                    if (!okw) {
                        fail = true;
                        break;
                    }
                    acc -= v * xv;
                }
            }
            for (int o = L >> 1; o >= 1; o >>= 1) acc += __shfl_down_sync(smask, acc, o, L);
            const bool seg_fail = __any_sync(smask, fail);
            if (act && sl == 0 && !seg_fail) {
                T val = publishable(acc * piv);
                xs[loc] = val;
                publish<T, OUT>(x, x64, q.r, val);
            }
            if (__any_sync(0xffffffffu, seg_fail)) {
                if (lane == 0) abort_flag = 1;
                break;
            }
        }
        __syncthreads();
        if (abort_flag) return;
    }
}

// nrhs right-hand sides (row-major n x K).  kp = power of two >= K lanes per
// row, 32/kp rows per task; lane k of a row owns right-hand side k.
template <class M, typename T, typename BT, int OUT>
__global__ void __launch_bounds__(512) k_sptrsv_mrhs(M m, int npos, int K, int kp, const BT* __restrict__ b, T* x,
                                                     double* x64, DevStatus* st, unsigned long long budget,
                                                     unsigned backoff)
{
    const int lane = threadIdx.x & 31;
    const int R = 32 / kp;
    const int seg = lane / kp, k = lane & (kp - 1);
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    const int ntasks = (npos + R - 1) / R;
    for (int t = gw; t < ntasks; t += nw) {
        int pos = t * R + seg;
        bool act = pos < npos && k < K;
        bool fail = false;
        if (act) {
            RowRef q = m.row(pos);
            T piv = (T)1 / (T)m.diag(q);
            T acc = (T)b[(size_t)q.r * K + k];
            for (int p = q.s; p < q.e; p++) {
                int c = m.c(p);
                T v = (T)m.v(p);
                T xv;
                if (!wait_ready(x + (size_t)c * K + k, xv, st, budget, q.r, backoff)) {
                    fail = true;
                    break;
                }
                acc -= v * xv;
            }
            if (!fail) publish<T, OUT>(x, x64, (size_t)q.r * K + k, acc * piv);
        }
        if (__any_sync(0xffffffffu, fail)) return;
    }
}

// FP64 residual r = b - L x over a plan layout (columns must be global);
// L lanes per row (single RHS) or one lane per right-hand side (K > 1).
template <typename RT>
__global__ void __launch_bounds__(256) k_residual(PermMat<double> m, int npos, int L, const double* __restrict__ b,
                                                  const double* __restrict__ x, RT* __restrict__ r)
{
    const int lane = threadIdx.x & 31;
    const int R = 32 / L, seg = lane / L, sl = lane & (L - 1);
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long ntasks = ((long long)npos + R - 1) / R;
    for (long long t = gw; t < ntasks; t += nw) {
        long long pos = t * R + seg;
        bool act = pos < npos;
        double acc = 0;
        RowRef q;
        if (act) {
            q = m.row((int)pos);
            if (sl == 0) acc = b[q.r] - m.diag(q) * x[q.r];
            for (int p = q.s + sl; p < q.e; p += L) acc -= m.v(p) * x[m.c(p)];
        }
        for (int o = L >> 1; o >= 1; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, L);
        if (act && sl == 0) r[q.r] = (RT)acc;
    }
}

template <typename RT>
__global__ void __launch_bounds__(256) k_residual_mrhs(PermMat<double> m, int npos, int K, int kp,
                                                       const double* __restrict__ b, const double* __restrict__ x,
                                                       RT* __restrict__ r)
{
    const int lane = threadIdx.x & 31;
    const int R = 32 / kp, seg = lane / kp, k = lane & (kp - 1);
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long ntasks = ((long long)npos + R - 1) / R;
    for (long long t = gw; t < ntasks; t += nw) {
        long long pos = t * R + seg;
        if (pos < npos && k < K) {
            RowRef q = m.row((int)pos);
            size_t ri = (size_t)q.r * K + k;
            double acc = b[ri] - m.diag(q) * x[ri];
            for (int p = q.s; p < q.e; p++) acc -= m.v(p) * x[(size_t)m.c(p) * K + k];
            r[ri] = (RT)acc;
        }
    }
}

}  // namespace sptrsv
