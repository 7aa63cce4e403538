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
// level at most U entries per lane); step t is one fixed-size record:
//   int   hdr[4]          kp, level_end (1 on a level's last step), 0, 0
//   T     val[U][32]      entry u of lane j (0 for an unused entry)
//   u16   slot[U][32]     its column's ring slot (slot R holds a constant 0)
//   u16   oslot[32]       ring slot of the lane's row (lanes with sub-lane 0)
//   int   xidx[32]        where x of the row goes (-1: nowhere, a warm-up row)
//   T     inv[32]         1 / L_rr
//   T     bv[32]          b of the row, written before each solve by
//                         k_band_gather from bidx (the row whose b it is)
// padded to 16 bytes.  The records of CH consecutive steps are one
// contiguous chunk; lane 0 brings chunks into NST shared-memory stages with
// cp.async.bulk (the bulk-copy engine, completion counted on an mbarrier),
// NST - 1 chunks ahead of the warp.  The waits on the mbarriers are bounded
// like every other wait of the library.
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

int rec_bytes(int U, int tsz)
{
    int b = 16 + U * 32 * tsz + U * 32 * 2 + 32 * 2 + 32 * 4 + 32 * tsz + 32 * tsz;
    return (b + 15) & ~15;
}

struct RecView {
    int U, tsz;
    size_t off_val, off_slot, off_oslot, off_xidx, off_inv, off_bv;
    RecView(int U_, int tsz_) : U(U_), tsz(tsz_)
    {
        off_val = 16;
        off_slot = off_val + (size_t)U * 32 * tsz;
        off_oslot = off_slot + (size_t)U * 32 * 2;
        off_xidx = off_oslot + 64;
        off_inv = off_xidx + 128;
        off_bv = off_inv + (size_t)32 * tsz;
    }
};

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
__global__ void k_band_gather(unsigned char* rec, int rec_bytes, size_t off_bv, const int* __restrict__ bidx,
                              long long nslots, const BT* __restrict__ b)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nslots;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = bidx[i];
        T* bv = reinterpret_cast<T*>(rec + (size_t)(i >> 5) * rec_bytes + off_bv);
        bv[i & 31] = r >= 0 ? (T)b[r] : (T)0;
    }
}

// One step's record fields of this lane, in registers.
template <typename T, int U>
struct BandStep {
    int kp, lend, os, xi;
    T v[U], bv, inv;
    int sl[U];
    __device__ __forceinline__ void load(const unsigned char* r, int lane, size_t off_val, size_t off_slot,
                                         size_t off_oslot, size_t off_xidx, size_t off_inv, size_t off_bv)
    {
        const int4 hdr = *reinterpret_cast<const int4*>(r);
        kp = hdr.x;
        lend = hdr.y;
        const T* val = reinterpret_cast<const T*>(r + off_val);
        const unsigned short* slot = reinterpret_cast<const unsigned short*>(r + off_slot);
#pragma unroll
        for (int q = 0; q < U; q++) {
            v[q] = val[q * 32 + lane];
            sl[q] = slot[q * 32 + lane];
        }
        bv = reinterpret_cast<const T*>(r + off_bv)[lane];
        os = reinterpret_cast<const unsigned short*>(r + off_oslot)[lane];
        xi = reinterpret_cast<const int*>(r + off_xidx)[lane];
        inv = reinterpret_cast<const T*>(r + off_inv)[lane];
    }
};

template <typename T, int U, int OUT>
__global__ void __launch_bounds__(32) k_sptrsv_band(const unsigned char* __restrict__ rec, int rec_bytes,
                                                    const int* __restrict__ ustep, int nunits, int R, T* x,
                                                    double* x64, DevStatus* st, unsigned long long budget)
{
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ __align__(8) unsigned long long bars[kBandNST];
    const int lane = threadIdx.x;
    T* ring = reinterpret_cast<T*>(sm);
    unsigned char* stage = sm + (((size_t)(R + 1) * sizeof(T) + 15) & ~(size_t)15);
    const size_t chunk_bytes = (size_t)kBandCH * rec_bytes;
    const size_t off_val = 16, off_slot = off_val + (size_t)U * 32 * sizeof(T), off_oslot = off_slot + U * 64,
                 off_xidx = off_oslot + 64, off_inv = off_xidx + 128, off_bv = off_inv + 32 * sizeof(T);
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
            // the record of step j + 1 is read into registers before step j
            // touches the slots, so its loads are not held behind step j's
            // shared-memory store (the compiler cannot tell the two apart)
            BandStep<T, U> cur, nxt;
            cur.load(cb, lane, off_val, off_slot, off_oslot, off_xidx, off_inv, off_bv);
            for (int j = 0; j < steps; j++) {
                if (j + 1 < steps)
                    nxt.load(cb + (size_t)(j + 1) * rec_bytes, lane, off_val, off_slot, off_oslot, off_xidx, off_inv,
                             off_bv);
                // two partial sums halve the dependent multiply-add chain
                T a0 = cur.bv, a1 = (T)0;
#pragma unroll
                for (int q = 0; q < U; q += 2) {
                    a0 -= cur.v[q] * ring[cur.sl[q]];
                    if (q + 1 < U) a1 -= cur.v[q + 1] * ring[cur.sl[q + 1]];
                }
                T acc = a0 + a1;
                for (int o = cur.kp >> 1; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if ((lane & (cur.kp - 1)) == 0 && cur.os < R) {
                    const T xv = acc * cur.inv;
                    ring[cur.os] = xv;
                    if (cur.xi >= 0) {
                        if (x) x[cur.xi] = xv;
                        if (OUT == OUT_SET64) x64[cur.xi] = (double)xv;
                        if (OUT == OUT_ADD64) x64[cur.xi] += (double)xv;
                    }
                }
                if (cur.lend) __syncwarp();
                cur = nxt;
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
    kern<<<t.nunits, 32, smem, s>>>(rec, rb, t.ustep, t.nunits, t.R, x, x64, c->d_status, wait_budget_ns());
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
    const int rb64 = rec_bytes(U, 8), rb32 = rec_bytes(U, 4);
    std::vector<unsigned char> h64((size_t)ns * rb64, 0), h32((size_t)ns * rb32, 0);
    std::vector<int> bidx((size_t)ns * 32, -1);
    const RecView V64(U, 8), V32(U, 4);
    for (long long t = 0; t < ns; t++) {
        const Step& sp = steps[t];
        unsigned char* r64 = &h64[(size_t)t * rb64];
        unsigned char* r32 = &h32[(size_t)t * rb32];
        const int hdr[4] = {sp.kp, sp.level_end, sp.cnt, 0};
        memcpy(r64, hdr, 16);
        memcpy(r32, hdr, 16);
        auto* v64 = reinterpret_cast<double*>(r64 + V64.off_val);
        auto* v32 = reinterpret_cast<float*>(r32 + V32.off_val);
        auto* s64 = reinterpret_cast<unsigned short*>(r64 + V64.off_slot);
        auto* s32 = reinterpret_cast<unsigned short*>(r32 + V32.off_slot);
        auto* o64 = reinterpret_cast<unsigned short*>(r64 + V64.off_oslot);
        auto* o32 = reinterpret_cast<unsigned short*>(r32 + V32.off_oslot);
        auto* x64 = reinterpret_cast<int*>(r64 + V64.off_xidx);
        auto* x32 = reinterpret_cast<int*>(r32 + V32.off_xidx);
        auto* i64 = reinterpret_cast<double*>(r64 + V64.off_inv);
        auto* i32 = reinterpret_cast<float*>(r32 + V32.off_inv);
        for (int j = 0; j < 32; j++) {
            o64[j] = o32[j] = (unsigned short)R;  // no row: slot R is never written
            x64[j] = x32[j] = -1;
            for (int q = 0; q < U; q++) s64[q * 32 + j] = s32[q * 32 + j] = (unsigned short)R;
        }
        for (int w = 0; w < sp.cnt; w++) {
            const int r = all_order[sp.first + w];
            const int un = unit_of[r];
            const int lane0 = w * sp.kp;
            const int d = rp[r + 1] - 1;
            for (int q = rp[r]; q < d; q++) {
                const int k = q - rp[r];
                const int lane = lane0 + (k % sp.kp), uu = k / sp.kp;
                const int sl = slot_of[ci[q]];
                s64[uu * 32 + lane] = s32[uu * 32 + lane] = (unsigned short)sl;
                v64[uu * 32 + lane] = va[q];
                v32[uu * 32 + lane] = (float)va[q];
            }
            bool real = true;
            const int orow = outer_row(un, r, &real);
            o64[lane0] = o32[lane0] = (unsigned short)slot_of[r];
            x64[lane0] = x32[lane0] = real ? orow : -1;
            i64[lane0] = 1.0 / va[d];
            i32[lane0] = 1.0f / (float)va[d];
            bidx[(size_t)t * 32 + lane0] = orow;
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
        const RecView V(kBandU, 8);
        k_band_gather<double, double><<<g, 256, 0, s>>>(t.rec64, t.rb64, V.off_bv, t.bidx, nslots,
                                                        static_cast<const double*>(b));
        SPT_CUDA(cudaGetLastError());
        return band_launch_t<double, OUT_X>(t, t.rec64, t.rb64, static_cast<double*>(x), nullptr, s);
    }
    const RecView V(kBandU, 4);
    if (b_f32)
        k_band_gather<float, float><<<g, 256, 0, s>>>(t.rec32, t.rb32, V.off_bv, t.bidx, nslots,
                                                      static_cast<const float*>(b));
    else
        k_band_gather<float, double><<<g, 256, 0, s>>>(t.rec32, t.rb32, V.off_bv, t.bidx, nslots,
                                                       static_cast<const double*>(b));
    SPT_CUDA(cudaGetLastError());
    float* xf = static_cast<float*>(x);
    if (out_mode == OUT_SET64) return band_launch_t<float, OUT_SET64>(t, t.rec32, t.rb32, xf, x64, s);
    if (out_mode == OUT_ADD64) return band_launch_t<float, OUT_ADD64>(t, t.rec32, t.rb32, xf, x64, s);
    return band_launch_t<float, OUT_X>(t, t.rec32, t.rb32, xf, x64, s);
}

}  // namespace sptrsv
