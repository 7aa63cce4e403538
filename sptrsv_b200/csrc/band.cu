// band.cu — the BAND schedule: one warp per independent unit of rows, level
// by level, x in a shared-memory ring, records streamed in by bulk copies.
//
// A unit is a set of consecutive rows that depends on no row outside it:
// the whole matrix, or one block of a partitioned plan's block system.  One
// warp (one CTA of 32 threads) solves its unit alone, so no flag, poll or
// wait on another warp exists anywhere: the warp takes the unit's levels in
// order and, between levels, only a __syncwarp orders its shared-memory
// writes before the next level's reads.  The cost of a dependent step is a
// shared-memory load, U fused multiply-adds, a short shuffle reduction and
// a shared-memory store (about 100-150 cycles), against a cross-warp hop
// through L2 of about 0.4 us in the level-ordered kernels.  It suits units
// whose levels are narrow (banded matrices: about 16 rows per level).
//
// Records.  A unit's levels are cut into steps of at most 32/kp rows with
// kp lanes per row (the smallest power of two that gives every row of the
// level at most U = 4 entries per lane); step t is one fixed-size record
// holding, per lane, a packet of 16-byte pieces stored piece-major (see
// band_rec_bytes): the lane's 4 entry values and their columns' slots (slot
// R holds a constant 0 for unused entries), the slot and output row of the
// lane's row (-1: a warm-up row, x goes nowhere), 1 / L_rr, the step's kp
// and whether it ends its level, and b of the row, written before each solve
// by k_band_gather from bidx (the row whose b it is).  A lane reads its
// packet with 3-4 conflict-free 128-bit loads.  The records of CH
// consecutive steps are one contiguous chunk; lane 0 brings chunks into NST
// shared-memory stages with cp.async.bulk (the bulk-copy engine, completion
// counted on an mbarrier), NST - 1 chunks ahead of the warp.  The waits on
// the mbarriers are bounded like every other wait of the library.
//
// Slots.  A row's value lives in a shared-memory slot from its level until
// the last level that reads it.  The builder hands slots out in the warp's
// write order from a free list and takes a slot back at the first level past
// its occupant's last reader (interval allocation over the level order), so
// R = the most values alive at once (at most 8192); slot R holds 0 for
// unused entries.
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"
#include "plan.h"
#include "solve_kernels.cuh"

namespace sptrsv {

namespace {

constexpr int kBandCH = 16;       // steps per chunk
constexpr int kBandNST = 3;       // chunk stages in shared memory
constexpr int kBandMaxRing = 8192;

// Record of one step: per lane a packet of 16-byte pieces, stored piece-major
// (piece k of lane j at k * 512 + j * 16), so a warp reads a piece with one
// conflict-free 128-bit shared-memory load per lane.
//   FP64 (4 pieces): {v0, v1} {v2, v3} {slot0|slot1, slot2|slot3, os|kp<<16|lend<<24, xi} {inv, bv}
//   FP32 (3 pieces): {v0..v3} {slot0|slot1, slot2|slot3, os|kp<<16|lend<<24, xi} {inv, bv, 0, 0}
// (slots and os 16 bits each; kp and lend are the step's, the same in every lane)
__host__ __device__ constexpr int band_pieces(int tsz) { return tsz == 8 ? 4 : 3; }
__host__ __device__ constexpr int band_rec_bytes(int tsz) { return band_pieces(tsz) * 512; }
// byte offset of lane j's b inside a record
__host__ __device__ constexpr size_t band_bv_offset(int tsz, int j)
{
    return tsz == 8 ? 3 * 512 + (size_t)j * 16 + 8 : 2 * 512 + (size_t)j * 16 + 4;
}

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier; false when the budget ran
// out (recorded in the status word) or another kernel reported an error.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, DevStatus* st,
                                          unsigned long long budget, int row)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned it = 1;; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0) {
            if (ld_relaxed(&st->code) != 0) return false;
            if (global_ns() - t0 > budget) {
                report(st, SPTRSV_ERR_TIMEOUT, row);
                return false;
            }
        }
    }
}

// b of every step's rows into the records (T = the record value type).
template <typename T, typename BT>
__global__ void k_band_gather(unsigned char* rec, const int* __restrict__ bidx, long long nslots,
                              const BT* __restrict__ b)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nslots;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = bidx[i];
        T* bv = reinterpret_cast<T*>(rec + (size_t)(i >> 5) * band_rec_bytes(sizeof(T)) +
                                     band_bv_offset(sizeof(T), (int)(i & 31)));
        *bv = r >= 0 ? (T)b[r] : (T)0;
    }
}

// One step's record pieces of this lane, as loaded (3-4 128-bit words), and
// unpacked into the fields the step uses (U = 4).
template <typename T>
struct BandRaw {
    static constexpr int NP = sizeof(T) == 8 ? 4 : 3;
    uint4 c[NP];
    __device__ __forceinline__ void fetch(const unsigned char* r, int lane)
    {
        const uint4* p = reinterpret_cast<const uint4*>(r) + lane;
#pragma unroll
        for (int k = 0; k < NP; k++) c[k] = p[32 * k];
    }
};

template <typename T>
struct BandStep {
    int kp, lend, os, xi;
    T v[4], bv, inv;
    int sl[4];
    __device__ __forceinline__ void unpack_meta(const uint4& c)
    {
        sl[0] = (int)(c.x & 0xffffu);
        sl[1] = (int)(c.x >> 16);
        sl[2] = (int)(c.y & 0xffffu);
        sl[3] = (int)(c.y >> 16);
        os = (int)(c.z & 0xffffu);
        kp = (int)((c.z >> 16) & 0xffu);
        lend = (int)(c.z >> 24);
        xi = (int)c.w;
    }
    __device__ __forceinline__ void unpack(const BandRaw<T>& r);
};
template <>
__device__ __forceinline__ void BandStep<double>::unpack(const BandRaw<double>& r)
{
    v[0] = __hiloint2double((int)r.c[0].y, (int)r.c[0].x);
    v[1] = __hiloint2double((int)r.c[0].w, (int)r.c[0].z);
    v[2] = __hiloint2double((int)r.c[1].y, (int)r.c[1].x);
    v[3] = __hiloint2double((int)r.c[1].w, (int)r.c[1].z);
    unpack_meta(r.c[2]);
    inv = __hiloint2double((int)r.c[3].y, (int)r.c[3].x);
    bv = __hiloint2double((int)r.c[3].w, (int)r.c[3].z);
}
template <>
__device__ __forceinline__ void BandStep<float>::unpack(const BandRaw<float>& r)
{
    v[0] = __uint_as_float(r.c[0].x);
    v[1] = __uint_as_float(r.c[0].y);
    v[2] = __uint_as_float(r.c[0].z);
    v[3] = __uint_as_float(r.c[0].w);
    unpack_meta(r.c[1]);
    inv = __uint_as_float(r.c[2].x);
    bv = __uint_as_float(r.c[2].y);
}

template <typename T, int U, int OUT>
__global__ void __launch_bounds__(32) k_sptrsv_band(const unsigned char* __restrict__ rec,
                                                    const int* __restrict__ ustep, int nunits, int R, T* x,
                                                    double* x64, DevStatus* st, unsigned long long budget)
{
    constexpr int rec_bytes = band_rec_bytes(sizeof(T));
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ __align__(8) unsigned long long bars[kBandNST];
    const int lane = threadIdx.x;
    T* ring = reinterpret_cast<T*>(sm);
    unsigned char* stage = sm + (((size_t)(R + 1) * sizeof(T) + 15) & ~(size_t)15);
    const size_t chunk_bytes = (size_t)kBandCH * rec_bytes;
    if (lane == 0) {
        for (int k = 0; k < kBandNST; k++) mbar_init(&bars[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    unsigned long long used = 0;  // chunks this CTA has consumed (stage = used % NST, parity from used / NST)
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int t0 = __ldg(ustep + u), t1 = __ldg(ustep + u + 1);
        const int nch = (t1 - t0 + kBandCH - 1) / kBandCH;
        if (lane == 0) ring[R] = (T)0;
        auto issue = [&](int c) {  // lane 0: chunk c of this unit into its stage
            const unsigned long long g = used + c;
            const int k = (int)(g % kBandNST);
            const int steps = min(kBandCH, t1 - t0 - c * kBandCH);
            const unsigned bytes = (unsigned)((size_t)steps * rec_bytes);
            mbar_expect_tx(&bars[k], bytes);
            bulk_g2s(stage + k * chunk_bytes, rec + (size_t)(t0 + c * kBandCH) * rec_bytes, bytes, &bars[k]);
        };
        if (lane == 0)
            for (int c = 0; c < min(nch, kBandNST - 1); c++) issue(c);
        __syncwarp();
        bool failed = false;
        int cfail = 0;
        for (int c = 0; c < nch; c++) {
            // keep NST - 1 chunks in flight: the stage of chunk c + NST - 1 was
            // last read at chunk c - 1 (the __syncwarp below ordered those reads;
            // the proxy fence orders them before the bulk copy's writes)
            if (lane == 0 && c + kBandNST - 1 < nch) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(c + kBandNST - 1);
            }
            const unsigned long long g = used + c;
            const int k = (int)(g % kBandNST);
            const unsigned parity = (unsigned)((g / kBandNST) & 1ull);
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&bars[k], parity, st, budget, u);
            if (!__shfl_sync(0xffffffffu, ok, 0)) {
                failed = true;
                cfail = c;
                break;
            }
            const unsigned char* cb = stage + k * chunk_bytes;
            const int steps = min(kBandCH, t1 - t0 - c * kBandCH);
            // Per step, in issue order: the next record's loads, this step's
            // slot loads, the next record's unpacking (its loads have landed by
            // then), the sums, the slot store.  So the chain from one level's
            // store to the next level's slot loads holds no other instruction.
            // A chunk's results stay in registers and go to x after its last
            // step, outside the level-to-level chain.
            BandStep<T> cur, nxt;
            BandRaw<T> raw;
            raw.fetch(cb, lane);
            cur.unpack(raw);
            T ov[kBandCH];
            int oi[kBandCH];
#pragma unroll
            for (int j = 0; j < kBandCH; j++) {
                oi[j] = -1;
                if (j < steps) {
                    if (j + 1 < steps) raw.fetch(cb + (size_t)(j + 1) * rec_bytes, lane);
                    T rv[U];
#pragma unroll
                    for (int q = 0; q < U; q++) rv[q] = ring[cur.sl[q]];
                    if (j + 1 < steps) nxt.unpack(raw);
                    // two partial sums halve the dependent multiply-add chain
                    T a0 = cur.bv, a1 = (T)0;
#pragma unroll
                    for (int q = 0; q < U; q += 2) {
                        a0 -= cur.v[q] * rv[q];
                        if (q + 1 < U) a1 -= cur.v[q + 1] * rv[q + 1];
                    }
                    T acc = a0 + a1;
                    for (int o = cur.kp >> 1; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                    if ((lane & (cur.kp - 1)) == 0 && cur.os < R) {
                        const T xv = acc * cur.inv;
                        ring[cur.os] = xv;
                        ov[j] = xv;
                        oi[j] = cur.xi;
                    }
                    if (cur.lend) __syncwarp();
                    cur = nxt;
                }
            }
#pragma unroll
            for (int j = 0; j < kBandCH; j++) {
                if (oi[j] >= 0) {
                    if (x) x[oi[j]] = ov[j];
                    if (OUT == OUT_SET64) x64[oi[j]] = (double)ov[j];
                    if (OUT == OUT_ADD64) x64[oi[j]] += (double)ov[j];
                }
            }
            __syncwarp();
        }
        if (failed) {
            // the chunks issued but not consumed, [cf, min(cf + NST, nch)), may
            // still be landing in shared memory: wait for them (bounded, 1 s)
            // before the CTA ends
            if (lane == 0) {
                const unsigned long long t_end = global_ns() + 1000000000ull;
                for (int c = cfail; c < min(cfail + kBandNST, nch); c++) {
                    const unsigned long long g = used + c;
                    const unsigned par = (unsigned)((g / kBandNST) & 1ull);
                    while (!mbar_try_wait(&bars[g % kBandNST], par) && global_ns() < t_end) {
                    }
                }
            }
            __syncwarp();
            return;
        }
        used += nch;
    }
}

template <typename T, int OUT>
int band_launch_t(const BandLayout& t, const unsigned char* rec, int rb, T* x, double* x64, cudaStream_t s)
{
    Ctx* c = ctx();
    auto kern = k_sptrsv_band<T, kBandU, OUT>;
    const size_t smem = (((size_t)(t.R + 1) * sizeof(T) + 15) & ~(size_t)15) + (size_t)kBandNST * kBandCH * rb;
    SPT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<t.nunits, 32, smem, s>>>(rec, t.ustep, t.nunits, t.R, x, x64, c->d_status, wait_budget_ns());
    SPT_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace

void band_free(BandLayout& t)
{
    cudaFree(t.rec64); cudaFree(t.rec32); cudaFree(t.bidx); cudaFree(t.ustep);
    t = BandLayout{};
}

int download_natural_csr(sptrsv_plan_s* p, std::vector<int>& rp, std::vector<int>& ci, std::vector<double>& va);

int build_band_layout(sptrsv_plan_s* p)
{
    if (p->band.rec64) return 0;
    const int n = p->n, U = kBandU;
    std::vector<int> rp, ci;
    std::vector<double> va;
    int e = download_natural_csr(p, rp, ci, va);
    if (e) return e;
    std::vector<int> lev(n);
    if (n > 0) SPT_CUDA(cudaMemcpy(lev.data(), p->levels, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    // units: the blocks of a block system, else the whole matrix
    std::vector<int> u0 = p->blk_starts;
    if (u0.empty()) u0.push_back(0);
    u0.push_back(n);
    const int nunits = (int)u0.size() - 1;
    // rows of the block system back to the outer plan's rows (partitioned plans)
    auto outer_row = [&](int unit, int r, bool* real) {
        if (p->part_tab.empty()) {
            *real = true;
            return r;
        }
        const int s = p->part_tab[4 * unit], a = p->part_tab[4 * unit + 1], base = p->part_tab[4 * unit + 3];
        const int o = s + (r - base);
        *real = o >= a;
        return o;
    };
    int maxoff = 0;
    for (int r = 0; r < n; r++) maxoff = std::max(maxoff, rp[r + 1] - rp[r] - 1);
    if (maxoff > 32 * U)
        return set_error(SPTRSV_ERR_UNSUPPORTED, "band schedule: a row holds %d off-diagonals, more than %d", maxoff,
                         32 * U);
    // last reader level of every row (0: never read)
    std::vector<int> lastread(n, 0);
    for (int r = 0; r < n; r++)
        for (int q = rp[r]; q < rp[r + 1] - 1; q++) lastread[ci[q]] = std::max(lastread[ci[q]], lev[r]);
    // rows of each unit by (level, row): the order the warp writes them
    std::vector<int> all_order(n);
    std::vector<int> ustep(nunits + 1, 0);
    std::vector<int> lbase(nunits), lcount(nunits);  // per unit: first level, levels
    std::vector<int> lcnt;                            // per unit and level: rows (prefix sums)
    std::vector<size_t> lcnt_off(nunits + 1, 0);
    for (int un = 0; un < nunits; un++) {
        const int a = u0[un], b = u0[un + 1];
        int lmin = 1 << 30, lmax = 0;
        for (int r = a; r < b; r++) {
            lmin = std::min(lmin, lev[r]);
            lmax = std::max(lmax, lev[r]);
        }
        const int nl = b > a ? lmax - lmin + 1 : 0;
        if (b > a && (b - a) > 128 * nl)
            return set_error(SPTRSV_ERR_UNSUPPORTED, "band schedule: levels hold %d rows on average, too wide for one "
                             "warp", (b - a) / nl);
        lbase[un] = lmin;
        lcount[un] = nl;
        lcnt_off[un + 1] = lcnt_off[un] + nl + 1;
        lcnt.resize(lcnt_off[un + 1], 0);
        int* cnt = &lcnt[lcnt_off[un]];
        for (int r = a; r < b; r++) cnt[lev[r] - lmin + 1]++;
        for (int l = 0; l < nl; l++) cnt[l + 1] += cnt[l];
        std::vector<int> pos(cnt, cnt + nl);
        for (int r = a; r < b; r++) all_order[a + pos[lev[r] - lmin]++] = r;
    }
    // shared-memory slots: a row's value lives from its write (its level)
    // to the last level that reads it.  Slots are handed out in the warp's
    // write order (all_order) from a free list; a slot returns to the list at
    // the first level past its occupant's last reader, so no value is lost
    // and R = the most values alive at once (a row nobody reads takes a slot
    // for its own level only)
    std::vector<int> slot_of(n, 0);
    int R = 1;
    {
        std::vector<int> freel;
        std::vector<std::vector<int>> release;  // per local level: slots free from the next level on
        for (int un = 0; un < nunits; un++) {
            const int a = u0[un], b = u0[un + 1];
            const int nl = lcount[un], lmin = lbase[un];
            freel.clear();
            release.assign(nl + 1, {});
            int top = 0, cur = -1;
            for (int q = a; q < b; q++) {
                const int r = all_order[q], L = lev[r] - lmin;
                while (cur < L) {  // entering a new level: recycle slots whose readers are done
                    if (cur >= 0)
                        for (int x : release[cur]) freel.push_back(x);
                    cur++;
                }
                int sl;
                if (!freel.empty()) {
                    sl = freel.back();
                    freel.pop_back();
                } else {
                    sl = top++;
                }
                slot_of[r] = sl;
                const int last = lastread[r] > 0 ? lastread[r] - lmin : L;  // level of its last reader
                release[last].push_back(sl);
            }
            R = std::max(R, top);
        }
        if (R > kBandMaxRing)
            return set_error(SPTRSV_ERR_UNSUPPORTED, "band schedule: %d values are alive at once, more than the %d "
                             "shared-memory slots", R, kBandMaxRing);
    }
    struct Step {
        int kp, level_end, first, cnt;  // rows all_order[first .. first + cnt)
    };
    std::vector<Step> steps;
    for (int un = 0; un < nunits; un++) {
        const int a = u0[un];
        const int* cnt = &lcnt[lcnt_off[un]];
        ustep[un] = (int)steps.size();
        for (int l = 0; l < lcount[un]; l++) {
            const int f = a + cnt[l], L = cnt[l + 1] - cnt[l];
            if (L == 0) continue;
            int mx = 0;
            for (int q = f; q < f + L; q++) {
                const int r = all_order[q];
                mx = std::max(mx, rp[r + 1] - rp[r] - 1);
            }
            int kp = 1;
            while ((mx + kp - 1) / kp > U) kp *= 2;
            const int per = 32 / kp;
            for (int q = 0; q < L; q += per) steps.push_back({kp, q + per >= L ? 1 : 0, f + q, std::min(per, L - q)});
        }
    }
    ustep[nunits] = (int)steps.size();
    // the unit of each row (for the ring slot base)
    std::vector<int> unit_of(n);
    for (int un = 0; un < nunits; un++)
        for (int r = u0[un]; r < u0[un + 1]; r++) unit_of[r] = un;
    const long long ns = (long long)steps.size();
    const int rb64 = band_rec_bytes(8), rb32 = band_rec_bytes(4);
    std::vector<unsigned char> h64((size_t)ns * rb64, 0), h32((size_t)ns * rb32, 0);
    std::vector<int> bidx((size_t)ns * 32, -1);
    for (long long t = 0; t < ns; t++) {
        const Step& sp = steps[t];
        unsigned char* r64 = &h64[(size_t)t * rb64];
        unsigned char* r32 = &h32[(size_t)t * rb32];
        // per lane: values, slots (R: the constant-0 slot), row slot, output row, 1/L_rr
        double v[32][4] = {};
        int sl[32][4], os[32], xi[32];
        double inv[32] = {};
        float invf[32] = {};
        for (int j = 0; j < 32; j++) {
            for (int q = 0; q < 4; q++) sl[j][q] = R;
            os[j] = R;  // no row: slot R is never written
            xi[j] = -1;
        }
        for (int w = 0; w < sp.cnt; w++) {
            const int r = all_order[sp.first + w];
            const int un = unit_of[r];
            const int lane0 = w * sp.kp;
            const int d = rp[r + 1] - 1;
            for (int q = rp[r]; q < d; q++) {
                const int k = q - rp[r];
                const int lane = lane0 + (k % sp.kp), uu = k / sp.kp;
                sl[lane][uu] = slot_of[ci[q]];
                v[lane][uu] = va[q];
            }
            bool real = true;
            const int orow = outer_row(un, r, &real);
            os[lane0] = slot_of[r];
            xi[lane0] = real ? orow : -1;
            inv[lane0] = 1.0 / va[d];
            invf[lane0] = 1.0f / (float)va[d];
            bidx[(size_t)t * 32 + lane0] = orow;
        }
        for (int j = 0; j < 32; j++) {
            const unsigned meta[4] = {(unsigned)sl[j][0] | ((unsigned)sl[j][1] << 16),
                                      (unsigned)sl[j][2] | ((unsigned)sl[j][3] << 16),
                                      (unsigned)os[j] | ((unsigned)sp.kp << 16) | ((unsigned)sp.level_end << 24),
                                      (unsigned)xi[j]};
            // FP64 pieces
            memcpy(r64 + 0 * 512 + j * 16, &v[j][0], 16);
            memcpy(r64 + 1 * 512 + j * 16, &v[j][2], 16);
            memcpy(r64 + 2 * 512 + j * 16, meta, 16);
            memcpy(r64 + 3 * 512 + j * 16, &inv[j], 8);
            // FP32 pieces
            const float vf[4] = {(float)v[j][0], (float)v[j][1], (float)v[j][2], (float)v[j][3]};
            memcpy(r32 + 0 * 512 + j * 16, vf, 16);
            memcpy(r32 + 1 * 512 + j * 16, meta, 16);
            memcpy(r32 + 2 * 512 + j * 16, &invf[j], 4);
        }
    }
    BandLayout t;
    t.U = U;
    t.R = R;
    t.nunits = nunits;
    t.nsteps = (int)ns;
    t.rb64 = rb64;
    t.rb32 = rb32;
    auto fail = [&](int code) {
        band_free(t);
        return code;
    };
    if (dalloc(&t.ustep, nunits + 1) != cudaSuccess || dalloc(&t.rec64, (long long)ns * rb64) != cudaSuccess ||
        dalloc(&t.rec32, (long long)ns * rb32) != cudaSuccess || dalloc(&t.bidx, ns * 32) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "band layout"));
    if (cudaMemcpy(t.ustep, ustep.data(), sizeof(int) * (size_t)(nunits + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
        (ns > 0 && (cudaMemcpy(t.rec64, h64.data(), h64.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
                    cudaMemcpy(t.rec32, h32.data(), h32.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
                    cudaMemcpy(t.bidx, bidx.data(), sizeof(int) * bidx.size(), cudaMemcpyHostToDevice) != cudaSuccess)))
        return fail(cuda_fail(cudaGetLastError(), "band layout upload"));
    p->band = t;
    return 0;
}

// One BAND solve: b (FP64 or FP32, indexed by the records' bidx) gathered
// into the records of the solve's precision, then one warp per unit.
// x (T) and x64 per out_mode; x may be null.
int band_solve(sptrsv_plan_s* p, bool f32, const void* b, bool b_f32, void* x, double* x64, int out_mode,
               cudaStream_t s)
{
    int e = build_band_layout(p);
    if (e) return e;
    const BandLayout& t = p->band;
    if (t.nsteps == 0) return 0;
    const long long nslots = (long long)t.nsteps * 32;
    const int g = grid_for(nslots, 256);
    if (!f32) {
        k_band_gather<double, double><<<g, 256, 0, s>>>(t.rec64, t.bidx, nslots, static_cast<const double*>(b));
        SPT_CUDA(cudaGetLastError());
        return band_launch_t<double, OUT_X>(t, t.rec64, t.rb64, static_cast<double*>(x), nullptr, s);
    }
    if (b_f32)
        k_band_gather<float, float><<<g, 256, 0, s>>>(t.rec32, t.bidx, nslots, static_cast<const float*>(b));
    else
        k_band_gather<float, double><<<g, 256, 0, s>>>(t.rec32, t.bidx, nslots, static_cast<const double*>(b));
    SPT_CUDA(cudaGetLastError());
    float* xf = static_cast<float*>(x);
    if (out_mode == OUT_SET64) return band_launch_t<float, OUT_SET64>(t, t.rec32, t.rb32, xf, x64, s);
    if (out_mode == OUT_ADD64) return band_launch_t<float, OUT_ADD64>(t, t.rec32, t.rb32, xf, x64, s);
    return band_launch_t<float, OUT_X>(t, t.rec32, t.rb32, xf, x64, s);
}

}  // namespace sptrsv
