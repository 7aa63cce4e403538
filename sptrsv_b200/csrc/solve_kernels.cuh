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
    int nnz;                      // entries of col/val; read only by kernels that check the CSR
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
    // piv = 1 / diag as the reference computes it (solve_csr_order.cu:239)
    __device__ __forceinline__ double inv(const RowRef& q) const { return 1.0 / __ldg(val + q.d); }
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
    const VT* __restrict__ di;      // [n] 1 / diagonal (rounded once, as 1/diag in VT)
    const int* __restrict__ seq;    // null: layout order; else natural -> position
    typedef VT V;
    __device__ __forceinline__ VT inv(const RowRef& q) const { return __ldg(di + q.d); }
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

// Per-lane state of one task.  Loaded one task ahead (software pipelining):
// the next task's row metadata, reciprocal diagonal, right-hand side and
// first element are in flight while the current task waits on its
// dependencies, so a warp that moves on only pays for the wait itself.
template <typename T>
struct Slot {
    int base, cnt, L;  // warp-uniform: first position, rows, lanes per row (0: diagonal-only rows)
    bool act;          // this lane's segment holds a row
    RowRef q;
    T piv;             // 1/diag (diagonal itself when L == 0)
    T acc;             // b for the segment's first lane, else 0
    int c0;            // first element of this lane (if q.s + sl < q.e)
    T v0;
};

template <class M, typename T, typename BT>
__device__ __forceinline__ void load_slot(Slot<T>& s, const M& m, int base, int cnt, int L, int lane,
                                          const BT* __restrict__ b)
{
    s.base = base;
    s.cnt = cnt;
    s.L = L;
    if (L == 0) {
        s.act = lane < cnt;
        if (s.act) {
            s.q = m.row(base + lane);
            s.piv = (T)m.diag(s.q);
            s.acc = (T)b[s.q.r];
        }
        return;
    }
    const int seg = lane / L, sl = lane & (L - 1);
    s.act = seg < cnt;
    if (s.act) {
        s.q = m.row(base + seg);
        s.piv = (T)m.inv(s.q);
        s.acc = sl == 0 ? (T)b[s.q.r] : (T)0;
        const int p = s.q.s + sl;
        if (p < s.q.e) {
            s.c0 = m.c(p);
            s.v0 = (T)m.v(p);
        }
    }
}

constexpr int kSlotU = 4;

// Runs one task: each lane takes its row's elements in rounds (lane sl of a
// row takes elements sl, sl+L, ...), the warp waits for a round's
// dependencies together, then rows reduce under their segment mask and
// publish.  Rows of one task are independent (tasks are level-aligned), so
// a warp-wide wait cannot deadlock.  Returns true (warp-uniform) on failure.
template <bool SMEM, class M, typename T, int OUT>
__device__ __forceinline__ bool run_slot(const Slot<T>& s, const M& m, int lane, T* x, double* x64, volatile T* xs,
                                         int cs, DevStatus* st, unsigned long long budget, unsigned backoff)
{
    if (s.L == 0) {  // diagonal-only rows: x = b / diag (solve_csr_multirow.cu:56-59)
        if (s.act) {
            T v = publishable(s.acc / s.piv);
            if (SMEM) xs[s.base + lane - cs] = v;
            publish<T, OUT>(x, x64, s.q.r, v);
        }
        return false;
    }
    const int L = s.L, seg = lane / L, sl = lane & (L - 1);
    const unsigned smask = segment_mask(L, seg);
    T acc = s.acc;
    const int mine = s.act ? max(0, (s.q.e - s.q.s - sl + L - 1) / L) : 0;
    const int rounds = __reduce_max_sync(0xffffffffu, mine);
    int p = s.q.s + sl;
    if (rounds > 0) {  // the first element was loaded with the task
        const bool have = 0 < mine;
        T xv = 0;
        if (!warp_wait<SMEM, T>(have, s.c0, x, xs, xv, st, budget, backoff, s.q.r)) return true;
        if (have) acc -= s.v0 * xv;
        p += L;
    }
    // long rows: kSlotU further elements per lane per wait, loads back to back
    for (int j = 1; j < rounds; j += kSlotU) {
        const int nh = min(kSlotU, mine - j);
        int cc[kSlotU];
        T vv[kSlotU], xv[kSlotU];
#pragma unroll
        for (int u = 0; u < kSlotU; u++) {
            cc[u] = 0;
            vv[u] = 0;
            if (u < nh) {
                cc[u] = m.c(p + u * L);
                vv[u] = (T)m.v(p + u * L);
            }
        }
        if (!warp_wait_n<SMEM, kSlotU, T>(nh, cc, x, xs, xv, st, budget, backoff, s.q.r)) return true;
#pragma unroll
        for (int u = 0; u < kSlotU; u++)
            if (u < nh) acc -= vv[u] * xv[u];
        p += kSlotU * L;
    }
    for (int o = L >> 1; o >= 1; o >>= 1) acc += __shfl_down_sync(smask, acc, o, L);
    if (s.act && sl == 0) {
        T val = publishable(acc * s.piv);
        if (SMEM) xs[s.base + seg - cs] = val;
        publish<T, OUT>(x, x64, s.q.r, val);
    }
    return false;
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
    auto load = [&](Slot<T>& s, int t) {
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
        load_slot(s, m, base, cnt, L, lane, b);
    };
    int t = gw;
    Slot<T> cur, nxt;
    if (t < ntasks) load(cur, t);
    while (t < ntasks) {
        const int tn = t + nw;
        if (tn < ntasks) load(nxt, tn);
        if (run_slot<false, M, T, OUT>(cur, m, lane, x, x64, nullptr, 0, st, budget, backoff)) return;
        cur = nxt;
        t = tn;
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
    for (int c = blockIdx.x; c < nclusters; c += gridDim.x) {
        const int cs = __ldg(cptr + c), cn = __ldg(cptr + c + 1) - cs;
        for (int i = threadIdx.x; i < cn; i += blockDim.x) xs[i] = sentinel_value<T>();
        if (threadIdx.x == 0) abort_flag = 0;
        __syncthreads();
        const int t1 = __ldg(ctask + c + 1);
        auto load = [&](Slot<T>& s, int t) {
            const int tb = __ldg(tbase + t);
            load_slot(s, m, tb, __ldg(tbase + t + 1) - tb, L, lane, b);
        };
        int t = __ldg(ctask + c) + wib;
        Slot<T> cur, nxt;
        if (t < t1) load(cur, t);
        while (t < t1) {
            const int tn = t + nwb;
            if (tn < t1) load(nxt, tn);
            if (run_slot<true, PermMat<V>, T, OUT>(cur, m, lane, x, x64, xs, cs, st, budget, backoff)) {
                if (lane == 0) abort_flag = 1;
                break;
            }
            cur = nxt;
            t = tn;
        }
        __syncthreads();
        if (abort_flag) return;
    }
}

// nrhs right-hand sides (row-major n x K), kp = power of two >= K lanes per
// row.  Level-aligned tasks of two kinds (table built by build_mrhs_tasks):
//
//   GROUP  {pos, cnt > 0, s0, lens[0..7], lens[8..15]}: the cnt <= E = 32/kp
//          short rows at positions [pos, pos+cnt), whose entries are the
//          contiguous range from s0; row j holds 4-bit lens[j] <= U entries.
//          Row seg takes lanes seg*kp .. seg*kp+kp-1; lane k owns right-hand
//          side k and handles all of its row's entries in one wait round.
//   PIECE  {pos, -npieces, e0, e1, pslot, cslot, piece}: entries [e0, e1) of
//          the long row at pos.  The warp's lanes are E element slots x kp
//          right-hand sides: slot e takes entries e0+e, e0+e+E, ..., U per
//          wait round, so each entry's K-wide line of x is one coalesced
//          gather; the slots' partial sums are added by shuffles.  A row of
//          one piece publishes x directly; otherwise each piece stores its
//          partial sums in pbuf[pslot] and bumps the row's counter
//          pcnt[cslot]; the piece that bumps it last adds all of the row's
//          partials in piece order (deterministic) and publishes x.
//
// The solve is bound by how many x gathers are in flight (the memory system,
// not the arithmetic, sets the pace), so the x values of a round are copied
// into the warp's shared-memory slots with cp.async: U = 16 gathers per lane
// in flight without holding registers for them.  A copied value equal to the
// sentinel (its row not published yet, or a stale line in L1) is re-polled
// with ld.relaxed.gpu and written back into its slot, and the products are
// then taken in entry order, so the sums are deterministic.  A long row
// costs about one wait round whatever its length, and pieces of a row sit in
// the same level, so their tasks never wait on each other.  The next task's
// record is loaded one task ahead.
struct MrhsTask {
    int pos, cnt, e0, e1;  // GROUP: e0 = s0, e1 = lens of rows 0..7; PIECE: entry range
    int pslot, cslot, piece, pad;  // GROUP: pslot = lens of rows 8..15
};

template <typename T>
__device__ __forceinline__ T ld_cg(const T* p)
{
    return __ldcg(p);
}

// This lane's entries of a task: first entry s, count n, stride (GROUP 1, PIECE E).
__device__ __forceinline__ void mrhs_lane_range(const int4& h, const int4& h2, int seg, int E, int& s, int& n,
                                                int& stride)
{
    if (h.y > 0) {
        const unsigned long long lens = (unsigned)h.w | ((unsigned long long)(unsigned)h2.x << 32);
        int off = 0;
        for (int i = 0; i < seg; i++) off += (int)((lens >> (4 * i)) & 15u);
        s = h.z + off;
        n = seg < h.y ? (int)((lens >> (4 * seg)) & 15u) : 0;
        stride = 1;
    } else {
        s = h.z + seg;
        n = s < h.w ? (h.w - s + E - 1) / E : 0;
        stride = E;
    }
}

template <typename T>
__device__ __forceinline__ void cp_async_ca(T* smem, const T* g)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(sa), "l"(g), "n"(sizeof(T)) : "memory");
}
// 16 bytes through L2 only (no L1 line that could go stale while a row is pending)
__device__ __forceinline__ void cp_async_cg16(void* smem, const void* g)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Gather modes of the multi-RHS solve.
enum { MRHS_LD = 0, MRHS_CA = 1, MRHS_CG = 2 };

// The gathers of one wait round: x[cc[u]*K + k] into xs[u*32 + lane] for the
// lane's nh entries.  CG (K * sizeof(T) a multiple of 16 bytes): lanes with
// k % (16/sizeof(T)) == 0 copy 16 bytes for themselves and the next lanes
// (same row, same entries) through L2; otherwise each lane copies its value.
template <typename T, int U, int GM>
__device__ __forceinline__ void mrhs_gather(const int (&cc)[U], int nh, const T* xk, int K, int k, T* xs, int lane)
{
    constexpr int VEC = 16 / sizeof(T);
    if (GM == MRHS_LD) {
        T v[U];
#pragma unroll
        for (int u = 0; u < U; u++)
            if (u < nh) v[u] = ld_relaxed(xk + (size_t)cc[u] * K);
#pragma unroll
        for (int u = 0; u < U; u++)
            if (u < nh) xs[u * 32 + lane] = v[u];
        return;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
        if (u < nh) {
            if (GM == MRHS_CG) {
                if ((k & (VEC - 1)) == 0) cp_async_cg16(xs + u * 32 + lane, xk + (size_t)cc[u] * K);
            } else {
                cp_async_ca(xs + u * 32 + lane, xk + (size_t)cc[u] * K);
            }
        }
    }
    cp_async_wait_all();
    __syncwarp();
}

// Re-polls (ld.relaxed.gpu) the lane's gathered values that still hold the
// sentinel, writes each into its slot once ready, then subtracts the
// products in entry order from acc.  Returns false (warp-uniform) on timeout
// or abort.
template <typename T, int U>
__device__ __forceinline__ bool mrhs_finish_round(const int (&cc)[U], const T (&vv)[U], int nh, const T* xk, int K,
                                                  T* xs, int lane, T& acc, DevStatus* st, unsigned long long budget,
                                                  unsigned backoff, int row)
{
    unsigned pend = 0;
#pragma unroll
    for (int u = 0; u < U; u++)
        if (u < nh && is_pending(xs[u * 32 + lane])) pend |= 1u << u;
    if (__any_sync(0xffffffffu, pend != 0)) {
        unsigned long long t0 = 0;
        unsigned it = 0;
        while (true) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                if ((pend >> u) & 1u) {
                    const T v = ld_relaxed(xk + (size_t)cc[u] * K);
                    if (!is_pending(v)) {
                        xs[u * 32 + lane] = v;
                        pend &= ~(1u << u);
                    }
                }
            }
            if (!__any_sync(0xffffffffu, pend != 0)) break;
            ++it;
            if (backoff && it > 8) __nanosleep(backoff);
            if ((it & 63u) == 0) {
                int stop = 0;
                if (lane == 0) {
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
#pragma unroll
    for (int u = 0; u < U; u++)
        if (u < nh) acc -= vv[u] * xs[u * 32 + lane];
    __syncwarp();  // the slots are reused by the next round
    return true;
}

template <class M, typename T, int U>
__device__ __forceinline__ void mrhs_load_round(const M& m, int s, int stride, int nh, int (&cc)[U], T (&vv)[U])
{
#pragma unroll
    for (int u = 0; u < U; u++) {
        cc[u] = 0;
        vv[u] = 0;
        if (u < nh) {
            cc[u] = m.c(s + u * stride);
            vv[u] = (T)m.v(s + u * stride);
        }
    }
}

template <typename V, typename T, typename BT, int OUT, int U, int GM>
__global__ void __launch_bounds__(256) k_sptrsv_mrhs(PermMat<V> m, int ntasks, const MrhsTask* __restrict__ tasks,
                                                     int K, int kp, const BT* __restrict__ b, T* x, double* x64,
                                                     T* pbuf, int* pcnt, DevStatus* st, unsigned long long budget,
                                                     unsigned backoff)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int seg = lane / kp, k = lane & (kp - 1), E = 32 / kp;
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    const bool kok = k < K;
    const T* xk = x + k;
    T* xs = reinterpret_cast<T*>(smem_raw) + (size_t)wib * U * 32;
    const int4* rec = reinterpret_cast<const int4*>(tasks);
    int t = gw;
    if (t >= ntasks) return;
    // Per task: record h/h2, this lane's entry range, row id and reciprocal
    // diagonal, and the first round's columns and values -- all issued at the
    // end of the previous task (or here for the first one).
    int4 h = __ldg(rec + 2 * (size_t)t), h2 = __ldg(rec + 2 * (size_t)t + 1);
    int s, n, stride;
    mrhs_lane_range(h, h2, seg, E, s, n, stride);
    int rr = __ldg(m.rowid + (h.y > 0 ? h.x + min(seg, h.y - 1) : h.x));
    T piv = (T)__ldg(m.di + (h.y > 0 ? h.x + min(seg, h.y - 1) : h.x));
    int cc[U];
    T vv[U];
    int nh = kok ? min(U, n) : 0;
    mrhs_load_round<PermMat<V>, T, U>(m, s, stride, nh, cc, vv);
    while (true) {
        const int tn = t + nw;
        int4 g = h, g2 = h2;
        if (tn < ntasks) {  // the next record, in flight while this task runs
            g = __ldg(rec + 2 * (size_t)tn);
            g2 = __ldg(rec + 2 * (size_t)tn + 1);
        }
        const bool group = h.y > 0;
        const bool out = group ? (seg < h.y && kok) : (seg == 0 && kok);
        const size_t xi = (size_t)rr * K + k;
        const T bval = out ? (T)b[xi] : (T)0;  // used at publish time
        T acc = 0;  // minus the sum of this lane's products
        mrhs_gather<T, U, GM>(cc, nh, xk, K, k, xs, lane);
        if (!mrhs_finish_round<T, U>(cc, vv, nh, xk, K, xs, lane, acc, st, budget, backoff, rr)) return;
        // later rounds (pieces cut longer than one round), loaded on the spot
        for (int j = U; __any_sync(FULL, kok && j < n); j += U) {
            const int mh = kok ? max(0, min(U, n - j)) : 0;
            mrhs_load_round<PermMat<V>, T, U>(m, s + j * stride, stride, mh, cc, vv);
            mrhs_gather<T, U, GM>(cc, mh, xk, K, k, xs, lane);
            if (!mrhs_finish_round<T, U>(cc, vv, mh, xk, K, xs, lane, acc, st, budget, backoff, rr)) return;
        }
        if (group) {
            if (out) publish<T, OUT>(x, x64, xi, (bval + acc) * piv);
        } else {
            for (int o = 16; o >= kp; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
            const int npieces = -h.y;
            if (npieces == 1) {
                if (out) publish<T, OUT>(x, x64, xi, (bval + acc) * piv);
            } else {
                if (out) pbuf[(size_t)h2.x * K + k] = acc;
                // the warp barrier orders the lanes' partial stores before lane
                // 0's acq_rel bump (release: they are visible to whoever sees
                // the bump; acquire: the last bumper sees every other piece's)
                __syncwarp();
                int last = 0;
                if (lane == 0) last = atom_add_acq_rel(pcnt + h2.y, 1) == npieces - 1;
                last = __shfl_sync(FULL, last, 0);
                __syncwarp();
                if (last) {
                    if (out) {
                        T sum = bval;
                        const size_t p0 = (size_t)(h2.x - h2.z) * K + k;
                        for (int q = 0; q < npieces; q++) sum += ld_cg(pbuf + p0 + (size_t)q * K);
                        publish<T, OUT>(x, x64, xi, sum * piv);
                    }
                }
            }
        }
        if (tn >= ntasks) break;
        // issue the next task's loads; they land while this warp moves on
        t = tn;
        h = g;
        h2 = g2;
        mrhs_lane_range(h, h2, seg, E, s, n, stride);
        const int rpos = h.y > 0 ? h.x + min(seg, h.y - 1) : h.x;
        rr = __ldg(m.rowid + rpos);
        piv = (T)__ldg(m.di + rpos);
        nh = kok ? min(U, n) : 0;
        mrhs_load_round<PermMat<V>, T, U>(m, s, stride, nh, cc, vv);
    }
}

// STRIP schedule (see strip.cu): warp w takes strips w, w + nw, ...; in a
// strip it solves chunk after chunk in wavefront order.  Lane j owns row j
// of the chunk at position P (slot P * 32 + j of the processing-order
// layout): it subtracts the row's entries outside the chunk (ring slots ~c
// from shared memory, other columns from x with the warp-convergent wait,
// kStripU per round), then the warp evaluates x_j = alpha_j + beta_j x_{j-1}
// by an affine Kogge-Stone scan: after the step of distance d lane j holds
// the composition of the maps j-2d+1..j, (alpha, beta) <- (alpha + beta *
// alpha', beta * beta') with (alpha', beta') from lane j - d; beta of the
// chunk's first row is 0, so the result is x_j.  A chunk's slot metadata is
// loaded two positions ahead and its entries and right-hand side one
// position ahead, so no load of the next chunk waits on another load.
template <typename V>
struct StripMat {
    const int* __restrict__ row;
    const int* __restrict__ pe;
    const int* __restrict__ ecol;
    const V* __restrict__ ev;
    const V* __restrict__ lsub;
    const V* __restrict__ di;
    const int* __restrict__ sptr;
};

constexpr int kStripU = 4;

template <typename T>
struct StripMeta {
    int row, e0, e1;
    int brow;  // row of b (row itself, except in a block system's streamed solve)
    T piv, lsub;
};

template <typename T, int U = kStripU>
struct StripEnt {
    T b;
    int cc[U];
    T vv[U];
};

template <typename V, typename T>
__device__ __forceinline__ void strip_meta(StripMeta<T>& z, const StripMat<V>& m, int slot)
{
    z.row = __ldg(m.row + slot);
    z.brow = z.row;
    z.e0 = __ldg(m.pe + slot);
    z.e1 = __ldg(m.pe + slot + 1);
    z.piv = (T)__ldg(m.di + slot);
    z.lsub = (T)__ldg(m.lsub + slot);
}

template <typename V, typename T, typename BT, int U = kStripU>
__device__ __forceinline__ void strip_ent(StripEnt<T, U>& z, const StripMeta<T>& md, const StripMat<V>& m,
                                          const BT* __restrict__ b, bool coherent_b = false)
{
    z.b = md.row >= 0 ? (T)(coherent_b ? ld_relaxed(b + md.brow) : b[md.brow]) : (T)0;
#pragma unroll
    for (int u = 0; u < U; u++) {
        z.cc[u] = 0;
        z.vv[u] = 0;
        if (md.e0 + u < md.e1) {
            z.cc[u] = __ldg(m.ecol + md.e0 + u);
            z.vv[u] = (T)__ldg(m.ev + md.e0 + u);
        }
    }
}

template <typename V, typename T, typename BT, int OUT>
__global__ void __launch_bounds__(512, 1) k_sptrsv_strip(StripMat<V> m, int nstrips, int W, const BT* __restrict__ b,
                                                      T* x, double* x64, DevStatus* st, unsigned long long budget,
                                                      unsigned backoff)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T* ring = reinterpret_cast<T*>(smem_raw) + (size_t)wib * W * 32;
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    for (int sidx = gw; sidx < nstrips; sidx += nw) {
        const int P0 = __ldg(m.sptr + sidx), P1 = __ldg(m.sptr + sidx + 1);
        StripMeta<T> m0, m1;
        StripEnt<T> e0;
        strip_meta<V, T>(m0, m, P0 * 32 + lane);
        strip_ent<V, T, BT>(e0, m0, m, b);
        if (P0 + 1 < P1) strip_meta<V, T>(m1, m, (P0 + 1) * 32 + lane);
        for (int P = P0; P < P1; P++) {
            const StripMeta<T> md = m0;
            const StripEnt<T> en = e0;
            if (P + 1 < P1) {
                m0 = m1;
                strip_ent<V, T, BT>(e0, m0, m, b);
                if (P + 2 < P1) strip_meta<V, T>(m1, m, (P + 2) * 32 + lane);
            }
            const int pos = P - P0;
            const int ec = md.e1 - md.e0;
            T acc = en.b;
            const int rounds = __reduce_max_sync(FULL, ec);
            for (int j = 0; j < rounds; j += kStripU) {
                const int nh = min(kStripU, ec - j);
                int cc[kStripU];
                T vv[kStripU], xv[kStripU];
#pragma unroll
                for (int u = 0; u < kStripU; u++) {
                    cc[u] = en.cc[u];
                    vv[u] = en.vv[u];
                    if (j > 0) {
                        cc[u] = 0;
                        vv[u] = 0;
                        if (u < nh) {
                            cc[u] = __ldg(m.ecol + md.e0 + j + u);
                            vv[u] = (T)__ldg(m.ev + md.e0 + j + u);
                        }
                    }
                }
                if (!warp_wait_n<true, kStripU, T>(nh, cc, x, ring, xv, st, budget, backoff, md.row)) return;
#pragma unroll
                for (int u = 0; u < kStripU; u++)
                    if (u < nh) acc -= vv[u] * xv[u];
            }
            T a = acc * md.piv, bb = -md.lsub * md.piv;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const T ap = __shfl_up_sync(FULL, a, d), bp = __shfl_up_sync(FULL, bb, d);
                if (lane >= d) {
                    a = a + bb * ap;
                    bb = bb * bp;
                }
            }
            const T xi = publishable(a);
            if (md.row >= 0) {
                ring[(pos % W) * 32 + lane] = xi;
                publish<T, OUT>(x, x64, md.row, xi);
            }
            __syncwarp();
        }
    }
}

// WAVE schedule (see strip.cu): CTA c takes the groups at places c,
// c + gridDim, ... of the processing order (gseq; natural order when null);
// warp w of the CTA solves line w of the group chunk by chunk (the same
// chunk arithmetic as STRIP).  The group's x values live in shared memory
// (filled with the sentinel first): a column inside the group is encoded
// ~(column - first row of the group) and polled there, so the wait on the
// line above is a shared-memory hop; other columns (the group's first line
// on the previous group, far planes) are polled in x.  After a group every
// warp meets at a CTA barrier before the shared copy is reused; a warp
// whose wait ran out raises a CTA flag there and the CTA leaves.
//
// Streamed host solves (bflag != nullptr): b arrives in segments of
// seg_rows rows while the kernel runs, each segment followed by its flag
// word set to `epoch`; a warp waits (acquire) for the flag of a row's
// segment before it loads that row's b (only when the row's segment differs
// from the last one the lane confirmed), and reads b coherently.  With hx
// set, the CTA also writes its group's x values from shared memory to that
// (mapped, pinned) host array in one burst once the group is done, so no
// store to host memory sits on the line-to-line critical path.
//
// U entries per lane are waited for together in one round; U = 2 when no
// row holds more than two entries outside its chunk recurrence (2D
// stencils), which shortens the poll loop and the dependent arithmetic on
// the line-to-line critical path (0.81 against 1.03 ms on a 2048 x 2048
// grid), else U = kStripU.  MULTI: some row holds more than U such entries
// (later rounds load theirs on the spot); STREAM: the streamed host solve.
template <typename V>
struct WaveMat {
    StripMat<V> c;                 // slot arrays (sptr unused)
    const int* __restrict__ runc;  // first chunk of each run
    const int* __restrict__ grun;  // first run of each group
    const int* __restrict__ grow;  // first row of each group
    const int* __restrict__ gseq;  // processing order of the groups (null: natural)
    // streamed solves of a block system (else null): per slot the outer row
    // whose b it takes, per group {outer row of its first row, its first row
    // that is not a warm-up row}
    const int* __restrict__ brow;
    const int* __restrict__ ghx;
};

template <typename V, typename T, typename BT, int OUT, int U, bool MULTI, bool STREAM>
__global__ void __launch_bounds__(512, 1) k_sptrsv_wave(WaveMat<V> w, int ngroups, const BT* __restrict__ b, T* x,
                                                        double* x64, DevStatus* st, unsigned long long budget,
                                                        unsigned backoff, const int* bflag, int seg_rows, int epoch,
                                                        double* hx)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int abort_flag;
    const unsigned FULL = 0xffffffffu;
    volatile T* xs = reinterpret_cast<volatile T*>(smem_raw);
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const StripMat<V>& m = w.c;
    if (threadIdx.x == 0) abort_flag = 0;
    int seg_ok = -1;  // streamed b: the last segment whose flag this lane saw set
    auto b_ready = [&](int row) -> bool {
        if (!STREAM) return true;
        const int sg = row >= 0 ? row / seg_rows : seg_ok;
        const bool need = bflag != nullptr && sg != seg_ok;
        if (!__any_sync(FULL, need)) return true;
        if (!warp_wait_flag(need, bflag + (need ? sg : 0), epoch, st, budget, row)) return false;
        if (need) seg_ok = sg;
        return true;
    };
    for (int k = blockIdx.x; k < ngroups; k += gridDim.x) {
        const int g = w.gseq ? __ldg(w.gseq + k) : k;
        const int r0 = __ldg(w.grow + g), nr = __ldg(w.grow + g + 1) - r0;
        for (int t = threadIdx.x; t < nr; t += blockDim.x) xs[t] = sentinel_value<T>();
        __syncthreads();
        const int run = __ldg(w.grun + g) + wib;
        bool failed = false;
        if (run < __ldg(w.grun + g + 1)) {
            const int q0 = __ldg(w.runc + run), q1 = __ldg(w.runc + run + 1);
            StripMeta<T> m0, m1;
            StripEnt<T, U> e0;
            strip_meta<V, T>(m0, m, q0 * 32 + lane);
            if (STREAM && w.brow && m0.row >= 0) m0.brow = __ldg(w.brow + q0 * 32 + lane);
            if (!b_ready(m0.row >= 0 ? m0.brow : -1)) failed = true;
            strip_ent<V, T, BT, U>(e0, m0, m, b, STREAM);
            if (q0 + 1 < q1) strip_meta<V, T>(m1, m, (q0 + 1) * 32 + lane);
            for (int q = q0; q < q1 && !failed; q++) {
                const StripMeta<T> md = m0;
                const StripEnt<T, U> en = e0;
                if (q + 1 < q1) {
                    m0 = m1;
                    if (STREAM && w.brow && m0.row >= 0) m0.brow = __ldg(w.brow + (q + 1) * 32 + lane);
                    if (!b_ready(m0.row >= 0 ? m0.brow : -1)) {
                        failed = true;
                        break;
                    }
                    strip_ent<V, T, BT, U>(e0, m0, m, b, STREAM);
                    if (q + 2 < q1) strip_meta<V, T>(m1, m, (q + 2) * 32 + lane);
                }
                const int ec = md.e1 - md.e0;
                T acc = en.b;
                const int rounds = MULTI ? __reduce_max_sync(FULL, ec) : 1;
                for (int j = 0; j < rounds; j += U) {
                    const int nh = min(U, ec - j);
                    int cc[U];
                    T vv[U], xv[U];
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        cc[u] = en.cc[u];
                        vv[u] = en.vv[u];
                        if (MULTI && j > 0) {
                            cc[u] = 0;
                            vv[u] = 0;
                            if (u < nh) {
                                cc[u] = __ldg(m.ecol + md.e0 + j + u);
                                vv[u] = (T)__ldg(m.ev + md.e0 + j + u);
                            }
                        }
                    }
                    if (!warp_wait_n<true, U, T>(nh, cc, x, xs, xv, st, budget, backoff, md.row)) {
                        failed = true;
                        break;
                    }
#pragma unroll
                    for (int u = 0; u < U; u++)
                        if (u < nh) acc -= vv[u] * xv[u];
                }
                if (failed) break;
                T a = acc * md.piv, bb = -md.lsub * md.piv;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const T ap = __shfl_up_sync(FULL, a, d), bp = __shfl_up_sync(FULL, bb, d);
                    if (lane >= d) {
                        a = a + bb * ap;
                        bb = bb * bp;
                    }
                }
                const T xi = publishable(a);
                if (md.row >= 0) {
                    xs[md.row - r0] = xi;
                    publish<T, OUT>(x, x64, md.row, xi);
                }
            }
        }
        if (failed && lane == 0) abort_flag = 1;
        __syncthreads();
        if (abort_flag) return;
        // each thread copies the slots it refills with the sentinel for the next group
        if (STREAM && hx) {
            const int o = w.ghx ? __ldg(w.ghx + 2 * g) : r0, t0 = w.ghx ? __ldg(w.ghx + 2 * g + 1) : 0;
            for (int t = t0 + threadIdx.x; t < nr; t += blockDim.x) hx[o + t] = (double)xs[t];
        }
    }
}

// Natural-order chunks (the plan's SIMPLE schedule): warp task t covers the
// natural rows [t*R, t*R+R) and solves them one after another with all 32
// lanes striding each row's elements.  A dependency inside the chunk was
// solved by this warp a moment ago and is read from the warp's shared-memory
// ring without waiting; others are polled warp-convergently.  The next row's
// metadata and first elements are loaded while the current row waits.
//
// CHECK (NatMat only; for callers whose CSR was never validated on the host):
// before a row's entries are touched, its range must satisfy
// 0 <= rowptr[r] < rowptr[r+1] <= nnz with the diagonal last
// (col[rowptr[r+1]-1] == r), and every off-diagonal column must satisfy
// 0 <= c < r before it indexes the ring or x.  A violation records
// SPTRSV_ERR_INVALID_CSR and the row in the status word and the warp leaves
// without any access through the bad index.
template <class M, typename T, typename BT, int OUT, bool CHECK = false>
__global__ void __launch_bounds__(512) k_sptrsv_chunk(M m, int n, int R, const BT* __restrict__ b, T* x, double* x64,
                                                      DevStatus* st, unsigned long long budget, unsigned backoff)
{
    __shared__ T ring[16][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T* my = ring[wib];
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
    const int ntasks = (n + R - 1) / R;
    for (int t = gw; t < ntasks; t += nw) {
        const int r0 = t * R, cnt = min(R, n - r0);
        // row j of the chunk: metadata in lane j (cnt <= 32)
        RowRef mq;
        mq.s = mq.e = 0;
        T mpiv = 0, mb = 0;
        bool bad = false;
        if (lane < cnt) {
            mq = m.row(r0 + lane);
            if constexpr (CHECK) bad = !(mq.s >= 0 && mq.s <= mq.e && mq.e < m.nnz) || m.c(mq.e) != mq.r;
            if (!bad) {
                mpiv = (T)m.inv(mq);
                mb = (T)b[mq.r];
            }
        }
        if constexpr (CHECK) {
            const unsigned badm = __ballot_sync(0xffffffffu, bad);
            if (badm) {
                if (lane == __ffs(badm) - 1) report(st, SPTRSV_ERR_INVALID_CSR, mq.r);
                return;
            }
        }
        int ns = __shfl_sync(0xffffffffu, mq.s, 0), ne = __shfl_sync(0xffffffffu, mq.e, 0);
        int nc = 0;
        T nv = 0;
        if (ns + lane < ne) {
            nc = m.c(ns + lane);
            nv = (T)m.v(ns + lane);
        }
        for (int j = 0; j < cnt; j++) {
            const int s = ns, e = ne;
            int c = nc;
            T v = nv;
            const T piv = __shfl_sync(0xffffffffu, mpiv, j);
            const T bj = __shfl_sync(0xffffffffu, mb, j);
            T acc = lane == 0 ? bj : (T)0;
            if (j + 1 < cnt) {  // prefetch the next row's first elements
                ns = __shfl_sync(0xffffffffu, mq.s, j + 1);
                ne = __shfl_sync(0xffffffffu, mq.e, j + 1);
                if (ns + lane < ne) {
                    nc = m.c(ns + lane);
                    nv = (T)m.v(ns + lane);
                }
            }
            for (int p = s + lane, first = 1; __any_sync(0xffffffffu, p < e); p += 32, first = 0) {
                const bool have = p < e;
                if (have && !first) {
                    c = m.c(p);
                    v = (T)m.v(p);
                }
                if constexpr (CHECK) {
                    const unsigned badm = __ballot_sync(0xffffffffu, have && (c < 0 || c >= r0 + j));
                    if (badm) {
                        if (lane == __ffs(badm) - 1) report(st, SPTRSV_ERR_INVALID_CSR, r0 + j);
                        return;
                    }
                }
                const bool local = have && c >= r0;
                T xv = local ? my[c - r0] : (T)0;
                if (!warp_wait<false, T>(have && !local, c, x, nullptr, xv, st, budget, backoff, r0 + j)) return;
                if (have) acc -= v * xv;
            }
            for (int o = 16; o >= 1; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                T val = publishable(acc * piv);
                my[j] = val;
                publish<T, OUT>(x, x64, (size_t)(r0 + j), val);
            }
            __syncwarp();
        }
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
