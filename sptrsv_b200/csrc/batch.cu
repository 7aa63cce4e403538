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
// A system whose levels hold few rows on average (n_s / nlevs_s below a
// threshold; a near-chain) gains nothing from the level order: every level
// costs a cross-warp hop through L2.  The hybrid schedule gives each such
// system to one warp of the same persistent launch, which walks it in natural
// order without any wait: the values of the most recent rows stay in a
// shared-memory ring, older ones are re-read from x (written by the same
// warp), and row metadata is loaded a chunk of 32 rows ahead.  The other
// systems keep the level-ordered tasks on the remaining warps.
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
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace sptrsv {
constexpr long long kSegChunk = 8192;  // elements per copy chunk of a partitioned batch
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
    // per-system level structure and the hybrid schedule
    int* lev = nullptr;          // [n] level of each union row (1-based)
    int* d_kplog = nullptr;      // [nsys] log2 of the right-hand-side class
    int* rblk_sys = nullptr;     // residual blocks: system of each 256-element block
    int* rblk_e0 = nullptr;      // and its first element inside the system
    int nrblk = 0;
    std::vector<int> row0h;      // [nsys+1] first union row of each system
    std::vector<int> sys_nlev;   // [nsys] levels of each system
    std::vector<int> sys_dist;   // [nsys] largest row - column distance of an entry
    std::vector<char> seq;       // [nsys] 1: solved by one warp in natural order (mode 2)
    int n_lvl = 0;               // rows in the level layout (the non-sequential systems)
    int* wptr = nullptr;         // [nseqw+1] per sequential warp: range in wsys
    int* wsys = nullptr;         // units in sequential-warp order: system
    int* wcol = nullptr;         // and right-hand side (-1: all of them)
    int nseqw = 0;
    double seq_width = 16.0;     // mode 2: sequential when n_s / nlevs_s < seq_width
    int mode = 2;                // 0: level-ordered tasks, 1: natural-order chunks, 2: hybrid
    int block_warps = 8, warps_per_sm = 0, backoff_ns = 0, ir_iters = 2;
    // partitioned batch (sptrsv_batch_set_partition): the block systems of the
    // long systems and the other systems whole, as a batch of their own; b is
    // gathered into its packed vectors and x scattered back, in chunks of at
    // most kSegChunk elements (gather chunks first, then scatter chunks)
    sptrsv_batch_s* inner = nullptr;
    int part_rows = 0;
    long long* d_seg = nullptr;  // [nseg * 3]: source offset, destination offset, length
    int nseg_g = 0, nseg_s = 0;
    double* pbx = nullptr;       // [inner->nvec] gathered right-hand sides
    double* pxx = nullptr;       // [inner->nvec] block-system solutions
    int part_systems = 0;        // systems cut into blocks
    long long part_warm = 0;     // warm-up rows in all
    double part_bound = 0;       // largest truncation bound of a block
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

// Systems solved by one warp each (hybrid schedule), over the natural-order
// union without diagonals.
struct SeqSet {
    const int* __restrict__ ptr;     // nptr
    const int* __restrict__ col;     // ncol
    const int* __restrict__ row0;    // [nsys+1]
    const int* __restrict__ sk;      // [nsys]
    const long long* __restrict__ soff;
    const int* __restrict__ wptr;    // [nseqw+1]
    const int* __restrict__ wsys;    // per unit: system
    const int* __restrict__ wcol;    // per unit: right-hand side (-1: all of them)
    int nseqw;
};

constexpr int kVkU = 8;         // elements per wait round in the level-ordered kernel
constexpr int kSeqRing = 1024;  // ring elements per sequential warp
constexpr int kSeqEC = 512;     // entries of one 32-row chunk that fit a stage buffer
constexpr int kSeqMaxK = 8;     // most right-hand sides one sequential warp carries (more: one warp per column)

__device__ __forceinline__ void cp_async(void* dst, const void* src, int bytes_is8)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (bytes_is8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared memory of one sequential warp: the ring of recent x values, then
// two stage buffers of one 32-row chunk each (relative row pointers, 1/diag,
// columns, values, right-hand sides).
template <typename V, typename T, typename BT>
struct SeqSmem {
    static constexpr size_t al(size_t x) { return (x + 15) & ~size_t(15); }
    static constexpr size_t ring = al(kSeqRing * sizeof(T));
    static constexpr size_t o_ptr = 0, o_di = al(33 * 4), o_col = o_di + al(32 * sizeof(V)),
                            o_val = o_col + al(kSeqEC * 4), o_b = o_val + al(kSeqEC * sizeof(V)),
                            buf = o_b + al(32 * kSeqMaxK * sizeof(BT));
    static constexpr size_t total = ring + 2 * buf;
};

// One warp solves system s (right-hand side col only, or all of them when
// col < 0) in natural order without waiting on anyone.
// Chunks of 32 rows are staged into shared memory with cp.async one chunk
// ahead (their row pointers are loaded two chunks ahead), so a row's work
// reads only shared memory: its entries, its right-hand sides and, for
// columns at most rw rows back, the ring of recent x values (slot = row mod
// rw).  An older column is read back from x, which this warp wrote.  Lane q
// owns right-hand side q (all of K > 1 columns, products subtracted in
// element order), or, for one column, lane j owns row j of each chunk (a
// sweep; the column's values are strided by K in b and x).  A chunk with
// more than kSeqEC entries is read from global memory instead.
template <typename V, typename T, typename BT, int OUT>
__device__ __forceinline__ void seq_system(const SeqSet& q, const V* __restrict__ val, const V* __restrict__ di,
                                           int s, int col, const BT* __restrict__ b, T* x, double* x64,
                                           unsigned char* region)
{
    using SM = SeqSmem<V, T, BT>;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int r0 = __ldg(q.row0 + s), r1 = __ldg(q.row0 + s + 1), K = __ldg(q.sk + s);
    const long long off = __ldg(q.soff + s);
    const int Ke = col >= 0 ? 1 : K;   // columns this warp carries
    const int c0 = col >= 0 ? col : 0; // first of them
    int kp = 1;
    while (kp < Ke) kp <<= 1;
    const int rw = kSeqRing / kp;
    const bool lk = lane < K;
    T* ring = reinterpret_cast<T*>(region);
    auto bufp = [&](int bi) { return region + SM::ring + (size_t)bi * SM::buf; };
    auto load_ptrs = [&](int cb, int& pl, int& pe) {
        const int cnt = min(32, r1 - cb);
        pl = lane < cnt ? __ldg(q.ptr + cb + lane) : 0;
        pe = __ldg(q.ptr + cb + cnt);
    };
    // issues the copies of chunk cb into buffer bi; returns whether its entries fit
    auto stage = [&](int bi, int cb, int pl, int pe, int& a_out) -> bool {
        const int cnt = min(32, r1 - cb);
        const int a = __shfl_sync(FULL, pl, 0);
        const int E = pe - a;
        unsigned char* base = bufp(bi);
        int* sptr = reinterpret_cast<int*>(base + SM::o_ptr);
        V* sdi = reinterpret_cast<V*>(base + SM::o_di);
        int* scol = reinterpret_cast<int*>(base + SM::o_col);
        V* sval = reinterpret_cast<V*>(base + SM::o_val);
        BT* sb = reinterpret_cast<BT*>(base + SM::o_b);
        if (lane < cnt) {
            sptr[lane] = pl - a;
            cp_async(sdi + lane, di + cb + lane, sizeof(V) == 8);
        }
        if (lane == 0) sptr[cnt] = E;
        const bool fits = E <= kSeqEC;
        if (fits)
            for (int p = lane; p < E; p += 32) {
                cp_async(scol + p, q.col + a + p, 0);
                cp_async(sval + p, val + a + p, sizeof(V) == 8);
            }
        const long long bo = off + (long long)(cb - r0) * K;
        if (Ke == 1)
            for (int p = lane; p < cnt; p += 32) cp_async(sb + p, b + bo + (long long)p * K + c0, sizeof(BT) == 8);
        else
            for (int p = lane; p < cnt * K; p += 32) cp_async(sb + p, b + bo + p, sizeof(BT) == 8);
        cp_async_commit();
        a_out = a;
        return fits;
    };
    int pl1 = 0, pe1 = 0, a_cur = 0, a_next = 0;
    load_ptrs(r0, pl1, pe1);
    bool fit_cur = stage(0, r0, pl1, pe1, a_cur);
    if (r0 + 32 < r1) load_ptrs(r0 + 32, pl1, pe1);
    cp_async_wait_all();
    __syncwarp();
    for (int c = 0, cb = r0; cb < r1; c++, cb += 32) {
        const int bi = c & 1;
        const int cnt = min(32, r1 - cb);
        bool fit_next = true;
        if (cb + 32 < r1) {
            fit_next = stage(bi ^ 1, cb + 32, pl1, pe1, a_next);
            if (cb + 64 < r1) load_ptrs(cb + 64, pl1, pe1);
        }
        const unsigned char* base = bufp(bi);
        const int* __restrict__ sptr = reinterpret_cast<const int*>(base + SM::o_ptr);
        const V* __restrict__ sdi = reinterpret_cast<const V*>(base + SM::o_di);
        const int* __restrict__ scol = reinterpret_cast<const int*>(base + SM::o_col);
        const V* __restrict__ sval = reinterpret_cast<const V*>(base + SM::o_val);
        const BT* __restrict__ sb = reinterpret_cast<const BT*>(base + SM::o_b);
        const int* gcol = q.col + a_cur;
        const V* gval = val + a_cur;
        if (Ke == 1) {
            // lane j owns row cb + j: first the entries before the chunk
            // (final values, a sorted prefix of the row), then a sweep over
            // the chunk in which row t's value is broadcast and every later
            // row holding column cb + t subtracts its product
            const int j = lane, i = cb + j;
            const bool own = j < cnt;
            T acc = own ? (T)sb[j] : (T)0;
            // the accumulated solution this correction adds to, loaded before the sweep
            const double old64 = (OUT == 2 && own) ? x64[off + (long long)(i - r0) * K + c0] : 0.0;
            const T piv = own ? (T)sdi[j] : (T)0;
            int p = own ? sptr[j] : 0;
            const int pe = own ? sptr[j + 1] : 0;
            int nc = 0x7fffffff;
            T nv = 0;
            for (; p < pe; p++) {
                const int cc = fit_cur ? scol[p] : __ldg(gcol + p);
                const T vv = (T)(fit_cur ? sval[p] : __ldg(gval + p));
                if (cc >= cb) {
                    nc = cc;
                    nv = vv;
                    break;
                }
                acc -= vv * ((i - cc <= rw) ? ring[cc & (rw - 1)] : __ldcg(x + off + (long long)(cc - r0) * K + c0));
            }
            T res = 0;
            for (int t = 0; t < cnt; t++) {
                const T mine = publishable(acc * piv);
                const T xt = __shfl_sync(FULL, mine, t);
                if (j == t) res = xt;
                if (nc == cb + t) {
                    acc -= nv * xt;
                    nc = 0x7fffffff;
                    if (++p < pe) {
                        nc = fit_cur ? scol[p] : __ldg(gcol + p);
                        nv = (T)(fit_cur ? sval[p] : __ldg(gval + p));
                    }
                }
            }
            if (own) {
                ring[i & (rw - 1)] = res;
                const long long xi = off + (long long)(i - r0) * K + c0;
                x[xi] = res;
                if (OUT == 1) x64[xi] = (double)res;
                if (OUT == 2) x64[xi] = old64 + (double)res;
            }
        } else {
            // lane q owns right-hand side q; rows one after another.  A row's
            // columns more than rw rows back (a sorted prefix, usually empty)
            // are read from x, the rest from the ring without a branch, four
            // at a time so their loads overlap.  The next row's pointers,
            // 1/diag and right-hand side are read one row ahead.
            if (lk) {
                T* __restrict__ rl = ring + lane;
                int e0 = sptr[0], e1 = sptr[1];
                T piv = (T)sdi[0], bj = (T)sb[lane];
                const long long xb = off + (long long)(cb - r0) * K + lane;  // x index of the chunk's first row
                double old64 = OUT == 2 ? x64[xb] : 0.0;  // the solution a correction adds to, a row ahead
                for (int j = 0; j < cnt; j++) {
                    const int i = cb + j;
                    int ne1 = 0;
                    T npiv = 0, nbj = 0;
                    double nold64 = 0.0;
                    if (j + 1 < cnt) {
                        ne1 = sptr[j + 2];
                        npiv = (T)sdi[j + 1];
                        nbj = (T)sb[(j + 1) * K + lane];
                        if (OUT == 2) nold64 = x64[xb + (long long)(j + 1) * K];
                    }
                    T acc = bj;
                    int p = e0;
                    if (fit_cur) {
                        for (; p < e1; p++) {  // columns beyond the ring
                            const int cc = scol[p];
                            if (i - cc <= rw) break;
                            acc -= (T)sval[p] * __ldcg(x + off + (long long)(cc - r0) * K + lane);
                        }
                        const int msk = rw - 1;
                        // four partial sums: the row's products are not one dependent chain
                        T acc1 = 0, acc2 = 0, acc3 = 0;
                        for (; p + 4 <= e1; p += 4) {
                            const int c0 = scol[p], c1 = scol[p + 1], c2 = scol[p + 2], c3 = scol[p + 3];
                            const T v0 = (T)sval[p], v1 = (T)sval[p + 1], v2 = (T)sval[p + 2], v3 = (T)sval[p + 3];
                            const T x0 = rl[(c0 & msk) * kp], x1 = rl[(c1 & msk) * kp], x2 = rl[(c2 & msk) * kp],
                                    x3 = rl[(c3 & msk) * kp];
                            acc -= v0 * x0;
                            acc1 -= v1 * x1;
                            acc2 -= v2 * x2;
                            acc3 -= v3 * x3;
                        }
                        for (; p < e1; p++) acc -= (T)sval[p] * rl[(scol[p] & msk) * kp];
                        acc += (acc1 + acc2) + acc3;
                    } else {
                        for (; p < e1; p++) {
                            const int cc = __ldg(gcol + p);
                            const T xc = (i - cc <= rw) ? rl[(cc & (rw - 1)) * kp]
                                                        : __ldcg(x + off + (long long)(cc - r0) * K + lane);
                            acc -= (T)__ldg(gval + p) * xc;
                        }
                    }
                    const T res = publishable(acc * piv);
                    rl[(i & (rw - 1)) * kp] = res;
                    const long long xi = off + (long long)(i - r0) * K + lane;
                    x[xi] = res;
                    if (OUT == 1) x64[xi] = (double)res;
                    if (OUT == 2) x64[xi] = old64 + (double)res;
                    e0 = e1;
                    e1 = ne1;
                    piv = npiv;
                    bj = nbj;
                    old64 = nold64;
                }
            }
        }
        cp_async_wait_all();
        __syncwarp();
        fit_cur = fit_next;
        a_cur = a_next;
    }
}

// Variable right-hand-side count, one lane per (row, right-hand side), over
// level-aligned tasks.  With sequential systems (q.nseqw > 0) the warps are
// numbered w = (warp in block) * gridDim + block; w < nseqw runs its
// sequential systems, the others take the level tasks round-robin.
template <typename V, typename T, typename BT, int OUT>
__global__ void __launch_bounds__(512, 1) k_sptrsv_vk(BatchMat bm, const V* __restrict__ val, const V* __restrict__ di,
                                                   int ntasks, const int* __restrict__ tbase,
                                                   const int* __restrict__ tkp, SeqSet q, const V* __restrict__ nval,
                                                   const V* __restrict__ ndi, const BT* __restrict__ b, T* x,
                                                   double* x64, DevStatus* st, unsigned long long budget,
                                                   unsigned backoff)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int w = wib * (int)gridDim.x + (int)blockIdx.x;
    if (w < q.nseqw) {  // w < nseqw implies wib < the sequential warps per block, each with its region
        for (int z = __ldg(q.wptr + w); z < __ldg(q.wptr + w + 1); z++)
            seq_system<V, T, BT, OUT>(q, nval, ndi, __ldg(q.wsys + z), __ldg(q.wcol + z), b, x, x64,
                                      smem_raw + (size_t)wib * SeqSmem<V, T, BT>::total);
        return;
    }
    const int gw = w - q.nseqw;
    const int nw = (int)(((long long)gridDim.x * blockDim.x) >> 5) - q.nseqw;
    for (int t = gw; t < ntasks; t += nw) {
        const int base = __ldg(tbase + t), cnt = __ldg(tbase + t + 1) - base, kp = __ldg(tkp + t);
        const int seg = lane / kp, k = lane & (kp - 1);
        const int pos = base + seg;
        const bool act = seg < cnt && k < __ldg(bm.krow + (seg < cnt ? pos : base));
        long long xr = 0;
        T acc = 0, piv = 0;
        int s = 0, len = 0;
        double old64 = 0.0;  // the solution a correction adds to, loaded with the task
        if (act) {
            xr = __ldg(bm.xrow + pos);
            acc = (T)b[xr + k];
            if (OUT == 2) old64 = x64[xr + k];
            piv = (T)__ldg(di + pos);
            s = __ldg(bm.ptr + pos);
            len = __ldg(bm.ptr + pos + 1) - s;
        }
        // rows of a task are in one level: the warp waits for each round of
        // kVkU elements together (loads issued back to back)
        const int rounds = __reduce_max_sync(0xffffffffu, len);
        for (int j = 0; j < rounds; j += kVkU) {
            const int nh = min(kVkU, len - j);
            long long xc[kVkU];
            T vv[kVkU], xv[kVkU];
#pragma unroll
            for (int u = 0; u < kVkU; u++) {
                xc[u] = 0;
                vv[u] = 0;
                if (u < nh) {
                    xc[u] = __ldg(bm.xdep + s + j + u) + k;
                    vv[u] = (T)__ldg(val + s + j + u);
                }
            }
            if (!warp_wait_n<false, kVkU, T>(nh, xc, x, nullptr, xv, st, budget, backoff, pos)) return;
#pragma unroll
            for (int u = 0; u < kVkU; u++)
                if (u < nh) acc -= vv[u] * xv[u];
        }
        if (act) {
            T r = publishable(acc * piv);
            st_relaxed(x + xr + k, r);
            if (OUT == 1) x64[xr + k] = (double)r;
            if (OUT == 2) x64[xr + k] = old64 + (double)r;
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

// r = b - L x in FP64 over the natural-order union (no dependencies), one
// thread per element of the packed vectors: block t covers the 256
// elements of system rblk_sys[t] starting at its element rblk_e0[t]
// (blocks never cross systems), element e of a system with K right-hand
// sides is (row e / K, column e mod K).  Threads of one row share its
// entries through L1; b, x and r are read and written coalesced.
__global__ void __launch_bounds__(256) k_residual_nat(const int* __restrict__ ptr, const int* __restrict__ col,
                                                      const double* __restrict__ val, const double* __restrict__ dg,
                                                      const int* __restrict__ rblk_sys, const int* __restrict__ rblk_e0,
                                                      const int* __restrict__ row0, const int* __restrict__ sk,
                                                      const long long* __restrict__ soff, const double* __restrict__ b,
                                                      const double* __restrict__ x, float* __restrict__ r)
{
    const int s = __ldg(rblk_sys + blockIdx.x);
    const int r0 = __ldg(row0 + s), n_s = __ldg(row0 + s + 1) - r0, K = __ldg(sk + s);
    const int e = __ldg(rblk_e0 + blockIdx.x) + threadIdx.x;
    if (e >= n_s * K) return;
    const int i = (int)(((double)e + 0.5) / (double)K);  // exact for e < 2^50
    const int k = e - i * K;
    const long long xb = __ldg(soff + s) + k - (long long)r0 * K;  // x[xb + c * K]: row c, right-hand side k
    const long long xe = __ldg(soff + s) + e;
    const int row = r0 + i;
    double acc = b[xe] - __ldg(dg + row) * x[xe];
    int p = __ldg(ptr + row);
    const int pe = __ldg(ptr + row + 1);
    for (; p + 4 <= pe; p += 4) {
        const int c0 = __ldg(col + p), c1 = __ldg(col + p + 1), c2 = __ldg(col + p + 2), c3 = __ldg(col + p + 3);
        const double v0 = __ldg(val + p), v1 = __ldg(val + p + 1), v2 = __ldg(val + p + 2), v3 = __ldg(val + p + 3);
        const double x0 = x[xb + (long long)c0 * K], x1 = x[xb + (long long)c1 * K], x2 = x[xb + (long long)c2 * K],
                     x3 = x[xb + (long long)c3 * K];
        acc -= v0 * x0;
        acc -= v1 * x1;
        acc -= v2 * x2;
        acc -= v3 * x3;
    }
    for (; p < pe; p++) acc -= __ldg(val + p) * x[xb + (long long)__ldg(col + p) * K];
    r[xe] = (float)acc;
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

// key = (level-1)*6 + log2(kp) per union row; rows of sequential systems get
// the key 6*nlevs, past every level, so they sort to the end of the layout
__global__ void k_batch_keys(const int* __restrict__ level, const int* __restrict__ sys_of_row,
                             const int* __restrict__ kp_log, const int* __restrict__ seqf, int nlevs, int n,
                             int* __restrict__ key, int* __restrict__ iota)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = sys_of_row[i];
        key[i] = seqf[s] ? 6 * nlevs : (level[i] - 1) * 6 + kp_log[s];
        iota[i] = i;
    }
}

__global__ void k_batch_rows(const int* __restrict__ order, const int* __restrict__ nptr, int n_lvl,
                             int* __restrict__ len)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= n_lvl; p += gridDim.x * blockDim.x) {
        if (p == n_lvl) {
            len[p] = 0;
            continue;
        }
        const int r = order[p];
        len[p] = nptr[r + 1] - nptr[r];
    }
}

// level layout positions p < n_lvl from the natural-order union
__global__ void k_batch_fill(const int* __restrict__ order, const int* __restrict__ nptr, const int* __restrict__ ncol,
                             const double* __restrict__ nval, const double* __restrict__ ndg,
                             const int* __restrict__ sys_of_row, const int* __restrict__ row0,
                             const long long* __restrict__ soff, const int* __restrict__ sk,
                             const int* __restrict__ ptr, int n_lvl, long long* __restrict__ xrow,
                             int* __restrict__ krow, long long* __restrict__ xdep, double* __restrict__ val64,
                             float* __restrict__ val32, double* __restrict__ dg64, double* __restrict__ di64,
                             float* __restrict__ di32)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_lvl; p += nw) {
        const int r = order[p];
        const int s = sys_of_row[r];
        const long long o = soff[s];
        const int k = sk[s], r0 = row0[s];
        const int a = nptr[r], e = nptr[r + 1], dst = ptr[p];
        for (int q = a + lane; q < e; q += 32) {
            const int c = ncol[q];
            xdep[dst + q - a] = o + (long long)(c - r0) * k;
            val64[dst + q - a] = nval[q];
            val32[dst + q - a] = (float)nval[q];
        }
        if (lane == 0) {
            const double d = ndg[r];
            xrow[p] = o + (long long)(r - r0) * k;
            krow[p] = k;
            dg64[p] = d;
            di64[p] = 1.0 / d;
            di32[p] = 1.0f / (float)d;
        }
    }
}

// largest row - column distance of each system (the first entry of a row has
// its smallest column; one block per system)
__global__ void k_sys_dist(const int* __restrict__ nptr, const int* __restrict__ ncol, const int* __restrict__ row0,
                           int nsys, int* __restrict__ out)
{
    __shared__ int red[32];
    for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
        int m = 0;
        for (int i = row0[s] + threadIdx.x; i < row0[s + 1]; i += blockDim.x)
            if (nptr[i + 1] > nptr[i]) m = max(m, i - ncol[nptr[i]]);
        m = __reduce_max_sync(0xffffffffu, m);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            int v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
            v = __reduce_max_sync(0xffffffffu, v);
            if (threadIdx.x == 0) out[s] = v;
        }
        __syncthreads();
    }
}

// levels of each system: the largest level among its rows (one block per system)
__global__ void k_sys_nlevs(const int* __restrict__ lev, const int* __restrict__ row0, int nsys, int* __restrict__ out)
{
    __shared__ int red[32];
    for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
        int m = 0;
        for (int i = row0[s] + threadIdx.x; i < row0[s + 1]; i += blockDim.x) m = max(m, lev[i]);
        m = __reduce_max_sync(0xffffffffu, m);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            int v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
            v = __reduce_max_sync(0xffffffffu, v);
            if (threadIdx.x == 0) out[s] = v;
        }
        __syncthreads();
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

void batch_free(sptrsv_batch_s* B);

void batch_part_free(sptrsv_batch_s* B)
{
    if (B->inner) {
        batch_free(B->inner);
        delete B->inner;
        B->inner = nullptr;
    }
    cudaFree(B->d_seg); cudaFree(B->pbx); cudaFree(B->pxx);
    B->d_seg = nullptr;
    B->pbx = B->pxx = nullptr;
    B->nseg_g = B->nseg_s = 0;
    B->part_rows = 0;
    B->part_systems = 0;
    B->part_warm = 0;
    B->part_bound = 0;
}

void batch_free(sptrsv_batch_s* B)
{
    batch_part_free(B);
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    if (B->cap_stream) cudaStreamDestroy(B->cap_stream);
    cudaFree(B->nptr); cudaFree(B->ncol); cudaFree(B->nval64); cudaFree(B->nval32); cudaFree(B->ndg64);
    cudaFree(B->ndi64); cudaFree(B->ndi32); cudaFree(B->tsys); cudaFree(B->tj); cudaFree(B->cdep);
    cudaFree(B->sys_row0); cudaFree(B->sys_chunk0); cudaFree(B->sys_k); cudaFree(B->sys_off); cudaFree(B->flags);
    cudaFree(B->row_sys); cudaFree(B->lev); cudaFree(B->d_kplog); cudaFree(B->wptr); cudaFree(B->wsys);
    cudaFree(B->wcol);
    cudaFree(B->rblk_sys); cudaFree(B->rblk_e0);
    cudaFree(B->ptr); cudaFree(B->xrow); cudaFree(B->krow); cudaFree(B->xdep); cudaFree(B->val64);
    cudaFree(B->val32); cudaFree(B->dg64); cudaFree(B->di64); cudaFree(B->di32); cudaFree(B->tbase);
    cudaFree(B->tkp); cudaFree(B->w32a); cudaFree(B->w32b);
}

// Level- and class-aligned tasks over the first n_lvl layout positions: a
// segment is one (level, kp) key and is cut into tasks of 32/kp rows;
// tkp[t] = kp of the task's segment.
int batch_tasks(sptrsv_batch_s* B, const int* key_sorted, int K, cudaStream_t s)
{
    int e = build_task_table(key_sorted, B->n_lvl, K, 0, &B->tbase, &B->ntasks, s);
    if (e) return e;
    SPT_CUDA(dalloc(&B->tkp, B->ntasks));
    if (B->ntasks > 0) {
        k_task_kp<<<grid_for(B->ntasks, 256), 256, 0, s>>>(B->tbase, B->ntasks, key_sorted, B->tkp);
        SPT_CUDA(cudaGetLastError());
    }
    return 0;
}

// (Re)builds the level layout for the systems not marked sequential in
// B->seq: order (level, rhs class), stable in the natural order.
int batch_level_layout(sptrsv_batch_s* B, cudaStream_t s)
{
    int** ip[] = {&B->ptr, &B->krow, &B->tbase, &B->tkp};
    for (int** p : ip) {
        cudaFree(*p);
        *p = nullptr;
    }
    cudaFree(B->xrow); cudaFree(B->xdep); cudaFree(B->val64); cudaFree(B->val32); cudaFree(B->dg64);
    cudaFree(B->di64); cudaFree(B->di32);
    B->xrow = B->xdep = nullptr;
    B->val64 = B->dg64 = B->di64 = nullptr;
    B->val32 = B->di32 = nullptr;
    B->ntasks = 0;
    const long long n = B->n;
    long long n_lvl = 0, m_lvl = 0;  // m_lvl: read back from the row pointer scan
    for (int k = 0; k < B->nsys; k++)
        if (!B->seq[k]) n_lvl += B->row0h[k + 1] - B->row0h[k];
    B->n_lvl = (int)n_lvl;
    int *d_seq = nullptr, *key = nullptr, *ord = nullptr, *kt = nullptr, *vt = nullptr, *scr = nullptr;
    auto cleanup = [&]() {
        cudaFree(d_seq); cudaFree(key); cudaFree(ord); cudaFree(kt); cudaFree(vt); cudaFree(scr);
    };
#define LCHK(call)                            \
    do {                                      \
        cudaError_t e_ = (call);              \
        if (e_ != cudaSuccess) {              \
            cleanup();                        \
            return cuda_fail(e_, #call);      \
        }                                     \
    } while (0)
    std::vector<int> seqi(B->seq.begin(), B->seq.end());
    LCHK(dalloc(&d_seq, B->nsys));
    LCHK(cudaMemcpy(d_seq, seqi.data(), sizeof(int) * (size_t)B->nsys, cudaMemcpyHostToDevice));
    LCHK(dalloc(&key, n));
    LCHK(dalloc(&ord, n));
    LCHK(dalloc(&kt, n));
    LCHK(dalloc(&vt, n));
    const long long sc1 = radix_scratch_ints(n), sc2 = scan_scratch_ints(n + 1);
    LCHK(dalloc(&scr, sc1 > sc2 ? sc1 : sc2));
    k_batch_keys<<<grid_for(n, 256), 256, 0, s>>>(B->lev, B->row_sys, B->d_kplog, d_seq, B->nlevs, (int)n, key, ord);
    LCHK(cudaGetLastError());
    LCHK(radix_sort_pairs(key, ord, kt, vt, n, 6 * B->nlevs, scr, s));
    LCHK(dalloc(&B->ptr, n_lvl + 1));
    k_batch_rows<<<grid_for(n_lvl + 1, 256), 256, 0, s>>>(ord, B->nptr, (int)n_lvl, B->ptr);
    LCHK(cudaGetLastError());
    LCHK(scan_exclusive(B->ptr, B->ptr, n_lvl + 1, scr, s));
    int mm = 0;
    LCHK(cudaMemcpyAsync(&mm, B->ptr + n_lvl, sizeof(int), cudaMemcpyDeviceToHost, s));
    LCHK(cudaStreamSynchronize(s));
    m_lvl = mm;
    LCHK(dalloc(&B->xrow, n_lvl));
    LCHK(dalloc(&B->krow, n_lvl));
    LCHK(dalloc(&B->xdep, m_lvl));
    LCHK(dalloc(&B->val64, m_lvl));
    LCHK(dalloc(&B->val32, m_lvl));
    LCHK(dalloc(&B->dg64, n_lvl));
    LCHK(dalloc(&B->di64, n_lvl));
    LCHK(dalloc(&B->di32, n_lvl));
    if (n_lvl > 0) {
        k_batch_fill<<<grid_for(n_lvl * 32, 256), 256, 0, s>>>(ord, B->nptr, B->ncol, B->nval64, B->ndg64,
                                                                B->row_sys, B->sys_row0, B->sys_off, B->sys_k,
                                                                B->ptr, (int)n_lvl, B->xrow, B->krow, B->xdep,
                                                                B->val64, B->val32, B->dg64, B->di64, B->di32);
        LCHK(cudaGetLastError());
    }
    {
        int e = batch_tasks(B, key, 6 * B->nlevs, s);
        if (e) {
            cleanup();
            return e;
        }
    }
    LCHK(cudaStreamSynchronize(s));
#undef LCHK
    cleanup();
    return 0;
}

constexpr int kModeLevel = 0, kModeChunk = 1, kModeHybrid = 2;
constexpr double kSeqAll = 1e9;  // a sequential width this large makes every system sequential
constexpr int kSeqSplitRows = 16384;  // sequential systems this long get one warp per right-hand side

// Sequential warps per block (warps 0.. of each block), each with its own
// shared-memory region; the other warps take the level tasks.
int seq_per_block(const sptrsv_batch_s* B) { return B->block_warps >= 8 ? 4 : B->block_warps >= 4 ? 2 : 1; }


// The level-ordered launch's grid size (every instantiation that a solve
// launches), before any sequential-warp assignment.
template <typename V, typename T, typename BT, int OUT>
int vk_grid(const sptrsv_batch_s* B, long long max_blocks, long long* g)
{
    const int cap = B->warps_per_sm > 0 ? (B->warps_per_sm + B->block_warps - 1) / B->block_warps : 0;
    const size_t smem = (size_t)seq_per_block(B) * SeqSmem<V, T, BT>::total;
    auto kern = k_sptrsv_vk<V, T, BT, OUT>;
    if (smem > 32 * 1024)  // the occupancy query needs the kernel's opt-in to large shared memory
        SPT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SPT_CUDA(persistent_grid(kern, 32 * B->block_warps, smem, max_blocks, cap, g));
    return 0;
}

long long vk_max_blocks(const sptrsv_batch_s* B, int nseqw)
{
    const long long a = div_up(B->ntasks, B->block_warps), c = div_up(nseqw, seq_per_block(B));
    return std::max(std::max(a, c), 1LL);
}

// Marks the sequential systems (mode 2: n_s / nlevs_s < seq_width and every
// dependency within the ring window: kSeqRing / kp rows, or kSeqRing rows for
// a system with more than kSeqMaxK right-hand sides or of at least
// kSeqSplitRows rows and several right-hand sides, which is solved one column
// per warp; or every system when seq_width >= kSeqAll),
// rebuilds the level layout when
// the set changed, and spreads the sequential systems
// over at most seq_per_block warps per block of the grid, largest first, each to the warp
// with the least work so far.
int batch_apply_schedule(sptrsv_batch_s* B, cudaStream_t s)
{
    std::vector<char> seq(B->nsys, 0);
    if (B->mode == kModeHybrid)
        for (int k = 0; k < B->nsys; k++) {
            const double nk = B->row0h[k + 1] - B->row0h[k];
            int kp = 1;
            while (kp < B->kk[k]) kp <<= 1;
            // a split system's units carry one column each: their ring spans kSeqRing rows
            const bool split = B->kk[k] > kSeqMaxK || (B->kk[k] > 1 && nk >= kSeqSplitRows);
            const bool fits = B->sys_dist[k] <= (split ? kSeqRing : kSeqRing / kp);
            seq[k] = B->seq_width >= kSeqAll || (fits && nk < B->seq_width * std::max(1, B->sys_nlev[k]));
        }
    if (seq != B->seq || !B->ptr) {
        B->seq = seq;
        int e = batch_level_layout(B, s);
        if (e) return e;
    }
    // units: a system with more than kSeqMaxK right-hand sides, or a long one
    // with several, becomes one unit per column (each swept by its own warp,
    // 0.13 us per row on a near-chain); other systems are one unit carrying
    // all their columns (0.4 us per row for K > 1)
    std::vector<std::pair<int, int>> list;
    for (int k = 0; k < B->nsys; k++) {
        if (!B->seq[k]) continue;
        const int nk = B->row0h[k + 1] - B->row0h[k];
        if (B->kk[k] > kSeqMaxK || (B->kk[k] > 1 && nk >= kSeqSplitRows))
            for (int c = 0; c < B->kk[k]; c++) list.push_back({k, c});
        else
            list.push_back({k, -1});
    }
    cudaFree(B->wptr);
    cudaFree(B->wsys);
    cudaFree(B->wcol);
    B->wptr = B->wsys = B->wcol = nullptr;
    B->nseqw = 0;
    if (list.empty()) return 0;
    long long g = 0, gmin = 1LL << 40;
    const long long mb = vk_max_blocks(B, (int)list.size());
    int e = vk_grid<double, double, double, 0>(B, mb, &g);
    if (e) return e;
    gmin = std::min(gmin, g);
    if ((e = vk_grid<float, float, double, 1>(B, mb, &g))) return e;
    gmin = std::min(gmin, g);
    if ((e = vk_grid<float, float, float, 2>(B, mb, &g))) return e;
    gmin = std::min(gmin, g);
    const int nw = (int)std::min<long long>((long long)list.size(), gmin * seq_per_block(B));
    auto work = [&](const std::pair<int, int>& u) {
        const double nk = B->row0h[u.first + 1] - B->row0h[u.first];
        return nk * (u.second >= 0 || B->kk[u.first] == 1 ? 1.0 : 3.0);
    };
    std::stable_sort(list.begin(), list.end(), [&](const std::pair<int, int>& a, const std::pair<int, int>& b2) {
        return work(a) > work(b2);
    });
    std::vector<std::vector<std::pair<int, int>>> per(nw);
    std::vector<double> load(nw, 0.0);
    for (const auto& u : list) {
        const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        per[w].push_back(u);
        load[w] += work(u);
    }
    std::vector<int> wp(nw + 1, 0), ws, wc;
    for (int w = 0; w < nw; w++) {
        for (const auto& u : per[w]) {
            ws.push_back(u.first);
            wc.push_back(u.second);
        }
        wp[w + 1] = (int)ws.size();
    }
    SPT_CUDA(dalloc(&B->wptr, nw + 1));
    SPT_CUDA(dalloc(&B->wsys, (long long)ws.size()));
    SPT_CUDA(dalloc(&B->wcol, (long long)wc.size()));
    SPT_CUDA(cudaMemcpy(B->wptr, wp.data(), sizeof(int) * wp.size(), cudaMemcpyHostToDevice));
    SPT_CUDA(cudaMemcpy(B->wsys, ws.data(), sizeof(int) * ws.size(), cudaMemcpyHostToDevice));
    SPT_CUDA(cudaMemcpy(B->wcol, wc.data(), sizeof(int) * wc.size(), cudaMemcpyHostToDevice));
    B->nseqw = nw;
    return 0;
}

template <typename V, typename T, typename BT, int OUT>
int batch_launch(sptrsv_batch_s* B, bool f32, const BT* b, T* x, double* x64, cudaStream_t s)
{
    Ctx* c = ctx();
    const int block = 32 * B->block_warps;
    const int cap = B->warps_per_sm > 0 ? (B->warps_per_sm + B->block_warps - 1) / B->block_warps : 0;
    if (B->mode == kModeChunk) {
        const V* val = f32 ? reinterpret_cast<const V*>(B->nval32) : reinterpret_cast<const V*>(B->nval64);
        const V* di = f32 ? reinterpret_cast<const V*>(B->ndi32) : reinterpret_cast<const V*>(B->ndi64);
        NatBatch nb{B->nptr, B->ncol, B->tsys, B->tj, B->cdep, B->sys_row0, B->sys_chunk0, B->sys_k, B->sys_off};
        SPT_CUDA(cudaMemsetAsync(B->flags, 0, sizeof(int) * (size_t)B->nchunks, s));
        auto kern = k_sptrsv_vkc<V, T, BT, OUT>;
        const size_t smem = (size_t)B->block_warps * 32 * 32 * sizeof(T);
        if (smem > 32 * 1024)
            SPT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        SPT_CUDA(launch_persistent_capped(kern, block, smem, div_up(B->nchunks, B->block_warps), cap, s, nb, val, di,
                                          B->nchunks, B->flags, b, x, x64, c->d_status, wait_budget_ns(),
                                          (unsigned)B->backoff_ns));
        return 0;
    }
    const V* val = f32 ? reinterpret_cast<const V*>(B->val32) : reinterpret_cast<const V*>(B->val64);
    const V* di = f32 ? reinterpret_cast<const V*>(B->di32) : reinterpret_cast<const V*>(B->di64);
    const V* nval = f32 ? reinterpret_cast<const V*>(B->nval32) : reinterpret_cast<const V*>(B->nval64);
    const V* ndi = f32 ? reinterpret_cast<const V*>(B->ndi32) : reinterpret_cast<const V*>(B->ndi64);
    BatchMat bm{B->ptr, B->xrow, B->krow, B->xdep};
    SeqSet q{B->nptr, B->ncol, B->sys_row0, B->sys_k, B->sys_off, B->wptr, B->wsys, B->wcol, B->nseqw};
    auto kern = k_sptrsv_vk<V, T, BT, OUT>;
    const size_t smem = B->nseqw > 0 ? (size_t)seq_per_block(B) * SeqSmem<V, T, BT>::total : 0;
    if (smem > 32 * 1024)
        SPT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (B->ntasks == 0 && B->nseqw == 0) return 0;
    SPT_CUDA(launch_persistent_capped(kern, block, smem, vk_max_blocks(B, B->nseqw), cap, s, bm, val, di, B->ntasks,
                                      (const int*)B->tbase, (const int*)B->tkp, q, nval, ndi, b, x, x64,
                                      c->d_status, wait_budget_ns(), (unsigned)B->backoff_ns));
    return 0;
}

int batch_residual(sptrsv_batch_s* B, const double* b, const double* x, cudaStream_t s)
{
    k_residual_nat<<<B->nrblk, 256, 0, s>>>(B->nptr, B->ncol, B->nval64, B->ndg64, B->rblk_sys, B->rblk_e0,
                                             B->sys_row0, B->sys_k, B->sys_off, b, x, B->w32b);
    SPT_CUDA(cudaGetLastError());
    return 0;
}

// Contiguous copies dst[d + t] = src[so + t], one block per table entry.
__global__ void __launch_bounds__(256) k_seg_copy(const long long* __restrict__ seg, const double* __restrict__ src,
                                                  double* __restrict__ dst)
{
    const long long* q = seg + 3 * (long long)blockIdx.x;
    const long long so = q[0], d = q[1], len = q[2];
    for (long long t = threadIdx.x; t < len; t += blockDim.x) dst[d + t] = src[so + t];
}

int batch_solve_impl(sptrsv_batch_s* B, const double* b, double* x, int precision, cudaStream_t s)
{
    if (B->n == 0) return 0;
    if (B->inner) {
        // partitioned: every refinement step runs on the block systems, whose
        // real rows equal the systems' rows to within the warm-up bound
        if (B->nseg_g) k_seg_copy<<<B->nseg_g, 256, 0, s>>>(B->d_seg, b, B->pbx);
        SPT_CUDA(cudaGetLastError());
        int e = batch_solve_impl(B->inner, B->pbx, B->pxx, precision, s);
        if (e) return e;
        if (B->nseg_s) k_seg_copy<<<B->nseg_s, 256, 0, s>>>(B->d_seg + 3LL * B->nseg_g, B->pxx, x);
        SPT_CUDA(cudaGetLastError());
        return 0;
    }
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
    return ::sptrsv::abi_guard([&]() -> int {
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
        int *d_sys = nullptr, *d_row0 = nullptr, *d_kplog = nullptr, *d_sk = nullptr;
        long long* d_soff = nullptr;
        auto cleanup = [&]() {
            cudaFree(U.ia); cudaFree(U.ja); cudaFree(U.a);
            cudaFree(d_sys); cudaFree(d_row0); cudaFree(d_kplog); cudaFree(d_sk); cudaFree(d_soff);
        };
        auto fail = [&](int code) {
            std::string msg = sptrsv_last_error_string();  // the public free below resets the last error
            cleanup();
            free_device_analysis(nullptr, &info);
            batch_free(B);
            delete B;
            return set_error(code, "%s", msg.c_str());
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
        // 2. levels of the union (validates every system's CSR too).  The level
        // kernel takes 32-row chunks system by system in order of their index
        // inside their system, so the dependency chains of all systems advance
        // together; in natural order a warp's chunk deep in one system's chain
        // holds up its later chunks of other systems (creating the 512-system
        // banded batch of up to 200,000 rows per system took 8.1 s, now 0.24 s).
        {
            int maxc = 0;
            for (int k = 0; k < nsys; k++) maxc = std::max(maxc, (mats[k].nr + 31) / 32);
            std::vector<int> tr0, tcnt;
            for (int c = 0; c < maxc; c++)
                for (int k = 0; k < nsys; k++)
                    if (c * 32 < mats[k].nr) {
                        tr0.push_back(row0[k] + c * 32);
                        tcnt.push_back(std::min(32, mats[k].nr - c * 32));
                    }
            int *d_tr0 = nullptr, *d_tcnt = nullptr;
            cudaError_t ce = dalloc(&d_tr0, (long long)tr0.size());
            if (ce == cudaSuccess) ce = dalloc(&d_tcnt, (long long)tcnt.size());
            if (ce == cudaSuccess)
                ce = cudaMemcpy(d_tr0, tr0.data(), sizeof(int) * tr0.size(), cudaMemcpyHostToDevice);
            if (ce == cudaSuccess)
                ce = cudaMemcpy(d_tcnt, tcnt.data(), sizeof(int) * tcnt.size(), cudaMemcpyHostToDevice);
            int e = ce != cudaSuccess ? cuda_fail(ce, "level tasks") : 0;
            if (!e) {
                const LevelTasks lt{d_tr0, d_tcnt, (long long)tr0.size()};
                e = run_analysis_impl(&info, &U, ORDER, &lt);
            }
            cudaFree(d_tr0);
            cudaFree(d_tcnt);
            if (e) return fail(e);
        }
        AnalysisRec* rec = find_analysis(info.row_ctr);
        B->nlevs = info.nlevs;
        // 3. per-system arrays
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
        // 4. levels kept per union row; levels of each system
        BCHK(dalloc(&B->lev, n));
        BCHK(cudaMemcpyAsync(B->lev, rec->d_levels, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s));
        {
            int* d_nl = nullptr;
            BCHK(dalloc(&d_nl, nsys));
            k_sys_nlevs<<<std::min(nsys, 4096), 256, 0, s>>>(B->lev, d_row0, nsys, d_nl);
            B->sys_nlev.assign(nsys, 0);
            cudaError_t ce = cudaGetLastError();
            if (ce == cudaSuccess)
                ce = cudaMemcpy(B->sys_nlev.data(), d_nl, sizeof(int) * (size_t)nsys, cudaMemcpyDeviceToHost);
            cudaFree(d_nl);
            BCHK(ce);
        }
        B->row0h = row0;
        {  // residual blocks: 256 consecutive packed elements of one system each
            std::vector<int> bs, be;
            for (int k = 0; k < nsys; k++) {
                const long long ne = (long long)mats[k].nr * nrhs[k];
                for (long long e0 = 0; e0 < ne; e0 += 256) {
                    bs.push_back(k);
                    be.push_back((int)e0);
                }
            }
            B->nrblk = (int)bs.size();
            BCHK(dalloc(&B->rblk_sys, B->nrblk));
            BCHK(dalloc(&B->rblk_e0, B->nrblk));
            BCHK(cudaMemcpy(B->rblk_sys, bs.data(), sizeof(int) * bs.size(), cudaMemcpyHostToDevice));
            BCHK(cudaMemcpy(B->rblk_e0, be.data(), sizeof(int) * be.size(), cudaMemcpyHostToDevice));
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
        {
            int* d_md = nullptr;
            BCHK(dalloc(&d_md, nsys));
            k_sys_dist<<<std::min(nsys, 4096), 256, 0, s>>>(B->nptr, B->ncol, d_row0, nsys, d_md);
            B->sys_dist.assign(nsys, 0);
            cudaError_t ce = cudaGetLastError();
            if (ce == cudaSuccess)
                ce = cudaMemcpy(B->sys_dist.data(), d_md, sizeof(int) * (size_t)nsys, cudaMemcpyDeviceToHost);
            cudaFree(d_md);
            BCHK(ce);
        }
        B->row_sys = d_sys;  // kept for the natural-order residual and the level layout
        d_sys = nullptr;
        B->d_kplog = d_kplog;
        d_kplog = nullptr;
        // 6. sequential systems and the level layout of the others (mode 2)
        {
            int e = batch_apply_schedule(B, s);
            if (e) return fail(e);
        }
        BCHK(dalloc(&B->w32a, B->nvec));
        BCHK(dalloc(&B->w32b, B->nvec));
        BCHK(cudaStreamSynchronize(s));
    #undef BCHK
        cleanup();
        free_device_analysis(nullptr, &info);
        *out = B;
        return ok();
    });
}

int sptrsv_batch_destroy(sptrsv_batch_t B)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B) return ok();
        batch_free(B);
        delete B;
        return ok();
    });
}

int sptrsv_batch_info(sptrsv_batch_t B, long long* offsets, int* n_total, int* nlevs, long long* vec_len)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B) return set_error(SPTRSV_ERR_INVALID_ARG, "batch_info: NULL");
        if (offsets) memcpy(offsets, B->off.data(), sizeof(long long) * (size_t)(B->nsys + 1));
        if (n_total) *n_total = B->n;
        if (nlevs) *nlevs = B->nlevs;
        if (vec_len) *vec_len = B->nvec;
        return ok();
    });
}

int sptrsv_batch_set_schedule(sptrsv_batch_t B, int mode, int block_warps, int warps_per_sm, int backoff_ns,
                              int ir_iters)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B || mode < kModeLevel || mode > kModeHybrid ||
            (block_warps != 2 && block_warps != 4 && block_warps != 8 && block_warps != 16) ||
            (mode == kModeChunk && block_warps > 8) || warps_per_sm < 0 || warps_per_sm > 64 || backoff_ns < 0 ||
            backoff_ns > 100000 || ir_iters < 0 || ir_iters > 16)
            return set_error(SPTRSV_ERR_INVALID_ARG, "batch_set_schedule: bad arguments");
        B->mode = mode;
        B->block_warps = block_warps;
        B->warps_per_sm = warps_per_sm;
        B->backoff_ns = backoff_ns;
        B->ir_iters = ir_iters;
        if (B->gexec) {  // the captured graph encodes the old schedule
            cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
        }
        int e = batch_apply_schedule(B, 0);
        if (!e && B->inner) e = sptrsv_batch_set_schedule(B->inner, mode, block_warps, warps_per_sm, backoff_ns, ir_iters);
        return e ? e : ok();
    });
}

int sptrsv_batch_set_seq_width(sptrsv_batch_t B, double width)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B || !(width >= 0.0) || width > 1e9) return set_error(SPTRSV_ERR_INVALID_ARG, "batch_set_seq_width: bad arguments");
        B->seq_width = width;
        if (B->gexec) {
            cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
        }
        int e = batch_apply_schedule(B, 0);
        if (!e && B->inner) e = sptrsv_batch_set_seq_width(B->inner, width);
        return e ? e : ok();
    });
}

int sptrsv_batch_seq_systems(sptrsv_batch_t B, int* nseq, int* nseq_warps, int* n_level_rows)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B) return set_error(SPTRSV_ERR_INVALID_ARG, "batch_seq_systems: NULL");
        if (B->inner) B = B->inner;  // a partitioned batch runs its block systems
        int c = 0;
        for (char f : B->seq) c += f ? 1 : 0;
        if (nseq) *nseq = c;
        if (nseq_warps) *nseq_warps = B->nseqw;
        if (n_level_rows) *n_level_rows = B->n_lvl;
        return ok();
    });
}

int sptrsv_batch_solve(sptrsv_batch_t B, const double* b, double* x, int precision, cudaStream_t s)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B || !b || !x || (precision != 32 && precision != 64))
            return set_error(SPTRSV_ERR_INVALID_ARG, "batch_solve: bad arguments");
        int e = batch_solve_impl(B, b, x, precision, s);
        return e ? e : ok();
    });
}

// Captures the whole solve (memsets, persistent solve launches, residuals) as
// a CUDA graph on first use for these (b, x, precision) and replays it on
// `s`; a different (b, x, precision) re-captures.
int sptrsv_batch_solve_graph(sptrsv_batch_t B, const double* b, double* x, int precision, cudaStream_t s)
{
    return ::sptrsv::abi_guard([&]() -> int {
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
    });
}

}  // extern "C"

namespace sptrsv {
int partition_blocks(const int* rp, const int* ci, const double* va, int n, int P, int threads, std::vector<int>& tab,
                     int* reach, double* bound, double min_ratio);
}

extern "C" {

// Cuts every system of at least 2 * block_rows rows (and whose rows are all
// diagonally dominant) into about n_s / block_rows blocks with warm-ups (the
// partitioned solve of the plan API: each block starts early from a zero
// boundary, the start chosen so that a proven bound on the dropped rows'
// effect is below 2^-60 relative to max|x|), and solves all blocks and the
// other systems as one batch.  block_rows = 0 returns to the plain batch.
int sptrsv_batch_set_partition(sptrsv_batch_t B, int block_rows)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B || block_rows < 0 || (block_rows > 0 && block_rows < 256))
            return set_error(SPTRSV_ERR_INVALID_ARG, "batch_set_partition: block_rows must be 0 or >= 256");
        if (B->gexec) {
            cudaGraphExecDestroy(B->gexec);
            B->gexec = nullptr;
        }
        if (block_rows == B->part_rows) return ok();
        batch_part_free(B);
        if (block_rows == 0) return ok();
        const int n = B->n, m = B->m, nsys = B->nsys;
        std::vector<int> nptr(n + 1), ncol(m > 0 ? m : 1);
        std::vector<double> nval(m > 0 ? m : 1), ndg(n);
        SPT_CUDA(cudaMemcpy(nptr.data(), B->nptr, sizeof(int) * (size_t)(n + 1), cudaMemcpyDeviceToHost));
        if (m > 0) {
            SPT_CUDA(cudaMemcpy(ncol.data(), B->ncol, sizeof(int) * (size_t)m, cudaMemcpyDeviceToHost));
            SPT_CUDA(cudaMemcpy(nval.data(), B->nval64, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost));
        }
        SPT_CUDA(cudaMemcpy(ndg.data(), B->ndg64, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
        // per system: its blocks (s, a, e) in local rows; one block [0, 0, n_s) when not cut
        std::vector<std::vector<int>> tabs(nsys);
        std::vector<double> bounds(nsys, 0.0);
        {
            const int nt = std::max(1u, std::thread::hardware_concurrency());
            std::vector<std::thread> th;
            for (int t = 0; t < nt; t++)
                th.emplace_back([&, t]() {
                    std::vector<int> rp, ci;
                    std::vector<double> va;
                    for (int sy = t; sy < nsys; sy += nt) {
                        const int r0 = B->row0h[sy], ns = B->row0h[sy + 1] - r0;
                        const int P = std::min(4096, ns / block_rows);
                        tabs[sy] = {0, 0, ns, 0};
                        if (P < 2) continue;
                        rp.assign(ns + 1, 0);
                        ci.clear();
                        va.clear();
                        for (int r = 0; r < ns; r++) {
                            for (int q = nptr[r0 + r]; q < nptr[r0 + r + 1]; q++) {
                                ci.push_back(ncol[q] - r0);
                                va.push_back(nval[q]);
                            }
                            ci.push_back(r);
                            va.push_back(ndg[r0 + r]);
                            rp[r + 1] = (int)ci.size();
                        }
                        std::vector<int> tab;
                        int w = 0;
                        double bnd = 0;
                        // blocks at least twice their warm-up, else the warm-ups would dominate
                        if (partition_blocks(rp.data(), ci.data(), va.data(), ns, P, 1, tab, &w, &bnd, 2.0) == 0) {
                            tabs[sy] = tab;
                            bounds[sy] = bnd;
                        }
                    }
                });
            for (auto& x : th) x.join();
        }
        // the block systems as device CSRs, and the copy tables
        std::vector<sp_mat_t> mats;
        std::vector<int> ks;
        std::vector<long long> gseg, sseg;
        auto add_chunks = [](std::vector<long long>& v, long long so, long long d, long long len) {
            for (long long o = 0; o < len; o += kSegChunk) {
                v.push_back(so + o);
                v.push_back(d + o);
                v.push_back(std::min<long long>(kSegChunk, len - o));
            }
        };
        auto free_mats = [&]() {
            for (auto& mm : mats) free_device_analysis(&mm, nullptr);
        };
        long long ioff = 0;
        int cut = 0;
        long long warm = 0;
        double bound = 0;
        std::vector<int> rp, ci;
        std::vector<double> va;
        for (int sy = 0; sy < nsys; sy++) {
            const int r0 = B->row0h[sy];
            const int k = B->kk[sy];
            const std::vector<int>& tab = tabs[sy];
            const int P = (int)tab.size() / 4;
            if (P > 1) {
                cut++;
                bound = std::max(bound, bounds[sy]);
            }
            for (int i = 0; i < P; i++) {
                const int s0 = tab[4 * i], a = tab[4 * i + 1], e = tab[4 * i + 2];
                warm += a - s0;
                rp.assign(e - s0 + 1, 0);
                ci.clear();
                va.clear();
                for (int r = s0; r < e; r++) {
                    for (int q = nptr[r0 + r]; q < nptr[r0 + r + 1]; q++)
                        if (ncol[q] - r0 >= s0) {
                            ci.push_back(ncol[q] - r0 - s0);
                            va.push_back(nval[q]);
                        }
                    ci.push_back(r - s0);
                    va.push_back(ndg[r0 + r]);
                    rp[r - s0 + 1] = (int)ci.size();
                }
                sp_mat_t mm{};
                int err = allocate_memory(rp.data(), ci.data(), va.data(), e - s0, &mm, ALL);
                if (err) {
                    free_mats();
                    return err;
                }
                mats.push_back(mm);
                ks.push_back(k);
                add_chunks(gseg, B->off[sy] + (long long)s0 * k, ioff, (long long)(e - s0) * k);
                add_chunks(sseg, ioff + (long long)(a - s0) * k, B->off[sy] + (long long)a * k, (long long)(e - a) * k);
                ioff += (long long)(e - s0) * k;
            }
        }
        sptrsv_batch_t in = nullptr;
        int err = sptrsv_batch_create((int)mats.size(), mats.data(), ks.data(), &in);
        free_mats();
        if (err) return err;
        B->inner = in;
        auto fail = [&](int code) {
            batch_part_free(B);
            return code;
        };
        err = sptrsv_batch_set_seq_width(in, B->seq_width);
        if (!err) err = sptrsv_batch_set_schedule(in, B->mode, B->block_warps, B->warps_per_sm, B->backoff_ns, B->ir_iters);
        if (err) return fail(err);
        if (gseg.size() / 3 > 0x7fffffffULL || sseg.size() / 3 > 0x7fffffffULL)
            return fail(set_error(SPTRSV_ERR_UNSUPPORTED, "batch_set_partition: too many copy chunks"));
        B->nseg_g = (int)(gseg.size() / 3);
        B->nseg_s = (int)(sseg.size() / 3);
        gseg.insert(gseg.end(), sseg.begin(), sseg.end());
        if (cudaMalloc((void**)&B->d_seg, sizeof(long long) * std::max<size_t>(1, gseg.size())) != cudaSuccess ||
            cudaMemcpy(B->d_seg, gseg.data(), sizeof(long long) * gseg.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMalloc((void**)&B->pbx, sizeof(double) * (size_t)in->nvec) != cudaSuccess ||
            cudaMalloc((void**)&B->pxx, sizeof(double) * (size_t)in->nvec) != cudaSuccess)
            return fail(cuda_fail(cudaGetLastError(), "batch_set_partition: buffers"));
        B->part_rows = block_rows;
        B->part_systems = cut;
        B->part_warm = warm;
        B->part_bound = bound;
        return ok();
    });
}

int sptrsv_batch_partition_info(sptrsv_batch_t B, int* systems_cut, int* inner_systems, long long* warm_rows,
                                double* bound)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!B) return set_error(SPTRSV_ERR_INVALID_ARG, "batch_partition_info: NULL");
        if (systems_cut) *systems_cut = B->inner ? B->part_systems : 0;
        if (inner_systems) *inner_systems = B->inner ? B->inner->nsys : B->nsys;
        if (warm_rows) *warm_rows = B->inner ? B->part_warm : 0;
        if (bound) *bound = B->inner ? B->part_bound : 0.0;
        return ok();
    });
}

}  // extern "C"
