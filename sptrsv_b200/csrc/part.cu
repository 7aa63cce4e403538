// part.cu — partitioned solves: row blocks solved independently after a
// warm-up, for row diagonally dominant matrices.
//
// L is cut into P blocks of consecutive rows; block i owns the real rows
// [a_i, e_i).  Solving block i on its own needs the x values of the rows
// before a_i, which are not known yet.  Instead the block starts its
// substitution K_i rows early, at s_i = a_i - K_i, with every entry that
// points before s_i dropped (a zero boundary), and keeps only its rows from
// a_i on.  The blocks then have no dependencies on each other: one
// block-diagonal system of n_ext = sum_i (e_i - s_i) rows, solved by a plan
// of its own with any schedule variant, its critical path about n/P + K rows
// deep instead of n.
//
// Why the warm-up is exact to 2^-60.  Let z be the block's solution from the
// zero boundary and d = x - z on rows r >= s.  Then
//     L_rr d_r = - sum_{s <= j < r} L_rj d_j - sum_{j < s} L_rj x_j,
// so, with X = max_{j < s} |x_j| <= max |x|, two bounds hold (both computed
// here at plan time, on the host, in FP64):
//   majorant  |d_r| <= E_r X,  E_r = (sum_{j<s} |L_rj| + sum_{s<=j<r} |L_rj| E_j) / |L_rr|
//             (the recurrence in absolute values; tight when the signs do
//             not cancel, e.g. stencils with same-sign neighbours);
//   spike     |d_r| <= (||Z_r||_1 + 4 (m+2) u E_r) X, where column c of Z is
//             the block's response to a unit value on column c < s
//             (Z_r = -(L_rc [c < s] + sum_{s<=j<r} L_rj Z_j) / L_rr), computed
//             in FP64 with rounding error below the second term (m: most
//             off-diagonals of a row, u = 2^-53); far tighter when signs
//             cancel (random values), and used when its dense rows are cheap
//             (coupled columns x most off-diagonals of a row <= 4096).
// Window argument: let w be the reach of L (most rows between an entry's
// column and its row).  A row r >= a + w depends only on rows in
// [r - w, r), all past s; with |L_rr| >= sum_j |L_rj| its bound is at most
// the largest bound among those rows.  So every real row of the block is
// bounded by the largest bound over its first w rows [a, a + w), and K is
// chosen (geometric search, then bisection) so that this is <= 2^-60: the
// dropped rows change x by less than 2^-60 max|x|, far below the rounding of
// the solve itself.  Block 0 starts at row 0 and is exact.
//
// Block starts a_i are put at "run starts" (rows that do not depend on the
// row before them: grid line starts), near i n / P, and so are the warm-up
// starts s_i, so a stencil's blocks hold whole grid lines.
#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

#include "internal.h"
#include "plan.h"
#include "solve_kernels.cuh"

namespace sptrsv {

namespace {

constexpr double kPartEps = 0x1p-60;
constexpr long long kSpikeMaxWork = 4096;  // coupled columns x most off-diagonals of a row

struct HostCsr {
    int n = 0;
    std::vector<int> rp, ci;
    std::vector<double> va;
};

// The plan's level layout back in natural row order (columns ascending, the
// diagonal last), on the host.
int download_natural(sptrsv_plan_s* p, HostCsr& h)
{
    const int n = p->n, m = p->nnz_off;
    std::vector<int> ptr(n + 1), rowid(n), col(m);
    std::vector<double> val(m), dg(n);
    SPT_CUDA(cudaMemcpy(ptr.data(), p->lev.ptr, sizeof(int) * (size_t)(n + 1), cudaMemcpyDeviceToHost));
    SPT_CUDA(cudaMemcpy(rowid.data(), p->lev.rowid, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    if (m > 0) {
        SPT_CUDA(cudaMemcpy(col.data(), p->lev.col, sizeof(int) * (size_t)m, cudaMemcpyDeviceToHost));
        SPT_CUDA(cudaMemcpy(val.data(), p->lev.val64, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost));
    }
    SPT_CUDA(cudaMemcpy(dg.data(), p->lev.dg64, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
    std::vector<int> pos(n);
    for (int q = 0; q < n; q++) pos[rowid[q]] = q;
    h.n = n;
    h.rp.assign(n + 1, 0);
    for (int r = 0; r < n; r++) h.rp[r + 1] = h.rp[r] + (ptr[pos[r] + 1] - ptr[pos[r]]) + 1;
    h.ci.resize(h.rp[n]);
    h.va.resize(h.rp[n]);
    for (int r = 0; r < n; r++) {
        const int q = pos[r], o = h.rp[r], len = ptr[q + 1] - ptr[q];
        for (int t = 0; t < len; t++) {
            h.ci[o + t] = col[ptr[q] + t];
            h.va[o + t] = val[ptr[q] + t];
        }
        h.ci[o + len] = r;
        h.va[o + len] = dg[q];
    }
    return 0;
}

// Largest bound over the window [a, min(e, a + w)) of a block started at s
// (see the file comment).  spike: also compute Z (W = min(w, s) columns).
double block_bound(const HostCsr& L, int s, int a, int e, int w, int maxoff, bool spike)
{
    if (s <= 0) return 0.0;  // starts at row 0: exact
    const int wend = std::min(e, a + w);
    const int rows = wend - s;
    std::vector<double> E(rows);
    const int W = std::min(w, s), c0 = s - W;
    const int ring = w + 1;
    std::vector<double> Z;
    std::vector<double> z;
    if (spike) {
        Z.assign((size_t)ring * W, 0.0);
        z.resize(W);
    }
    const double u = 0x1p-53, margin = 4.0 * (maxoff + 2) * u;
    double worst = 0;
    for (int r = s; r < wend; r++) {
        const int p0 = L.rp[r], p1 = L.rp[r + 1] - 1;
        const double dinv = 1.0 / std::fabs(L.va[p1]);
        double acc = 0;
        if (spike) std::fill(z.begin(), z.end(), 0.0);
        for (int p = p0; p < p1; p++) {
            const int c = L.ci[p];
            const double v = L.va[p];
            if (c < s) {
                acc += std::fabs(v);
                if (spike) z[c - c0] += v;
            } else {
                acc += std::fabs(v) * E[c - s];
                if (spike) {
                    const double* zc = &Z[(size_t)((c - s) % ring) * W];
                    for (int t = 0; t < W; t++) z[t] += v * zc[t];
                }
            }
        }
        E[r - s] = acc * dinv;
        double bnd = E[r - s];
        if (spike) {
            const double f = -1.0 / L.va[p1];
            double* zr = &Z[(size_t)((r - s) % ring) * W];
            double nrm = 0;
            for (int t = 0; t < W; t++) {
                zr[t] = z[t] * f;
                nrm += std::fabs(zr[t]);
            }
            bnd = std::min(bnd, nrm + margin * E[r - s]);
        }
        if (r >= a) worst = std::max(worst, bnd);
    }
    return worst;
}

// The nearest run start (a row that does not depend on the row before it)
// at or below r within `span` rows; r itself when there is none.
int run_start_below(const std::vector<unsigned char>& run0, int r, int span)
{
    for (int q = r; q >= 0 && q >= r - span; q--)
        if (run0[q]) return q;
    return r;
}

// Smallest warm-up start s for block [a, e) (searched from the guess K0).
// refine: doubling, then bisection (a search from scratch); otherwise the
// guess (a neighbouring block's warm-up) is tried at 9/10 and grown by 6/5
// until the bound holds.  Returns s (0 = exact) and the bound in *bnd.
int find_start(const HostCsr& L, const std::vector<unsigned char>& run0, int a, int e, int w, int maxoff,
               bool spike, int K0, double* bnd, bool refine = true)
{
    auto start_for = [&](long long K) {
        long long s = (long long)a - K;
        if (s <= 0) return 0;
        return run_start_below(run0, (int)s, w);
    };
    long long K = std::max<long long>(K0, w);
    if (!refine) {
        const long long Kd = std::max<long long>(w, K * 9 / 10);
        int sd = start_for(Kd);
        double bd = sd == 0 ? 0.0 : block_bound(L, sd, a, e, w, maxoff, spike);
        if (bd <= kPartEps) {
            *bnd = bd;
            return sd;
        }
        for (;;) {
            const int sk = start_for(K);
            const double bk = sk == 0 ? 0.0 : block_bound(L, sk, a, e, w, maxoff, spike);
            if (bk <= kPartEps) {
                *bnd = bk;
                return sk;
            }
            K = std::max<long long>(K * 6 / 5, K + w);
        }
    }
    int s = start_for(K);
    double b = block_bound(L, s, a, e, w, maxoff, spike);
    long long lo = 0, hi;
    if (b <= kPartEps) {
        hi = K;
        // one step down: a smaller warm-up may already do
        long long Kd = K * 4 / 5;
        if (Kd >= w) {
            int sd = start_for(Kd);
            double bd = block_bound(L, sd, a, e, w, maxoff, spike);
            if (bd <= kPartEps) {
                *bnd = bd;
                return sd;
            }
            lo = Kd;
        }
        *bnd = b;
        if (lo == 0) return s;
    } else {
        lo = K;
        for (;;) {
            K = std::max<long long>(K * 3 / 2, K + w);
            s = start_for(K);
            b = s == 0 ? 0.0 : block_bound(L, s, a, e, w, maxoff, spike);
            if (b <= kPartEps) break;
            lo = K;
        }
        hi = K;
    }
    int best_s = s;
    double best_b = b;
    for (int it = 0; it < 5 && hi - lo > w; it++) {
        const long long mid = (lo + hi) / 2;
        const int sm = start_for(mid);
        const double bm = sm == 0 ? 0.0 : block_bound(L, sm, a, e, w, maxoff, spike);
        if (bm <= kPartEps) {
            hi = mid;
            best_s = sm;
            best_b = bm;
        } else {
            lo = mid;
        }
    }
    *bnd = best_b;
    return best_s;
}

template <typename T>
__global__ void k_part_gather(const int* __restrict__ tab, const T* __restrict__ src, T* __restrict__ dst, int k)
{
    const int i = blockIdx.y;
    const long long s = tab[4 * i], e = tab[4 * i + 2], base = tab[4 * i + 3];
    const long long len = (e - s) * k;
    const T* from = src + s * k;
    T* to = dst + base * k;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < len; t += (long long)gridDim.x * blockDim.x)
        to[t] = from[t];
}

// x rows [a_i, e_i) from the block system's rows base_i + (a_i - s_i) ...
template <typename S, int MODE>
__global__ void k_part_scatter(const int* __restrict__ tab, const S* __restrict__ src, S* __restrict__ dst,
                               double* __restrict__ x64, int k)
{
    const int i = blockIdx.y;
    const long long s = tab[4 * i], a = tab[4 * i + 1], e = tab[4 * i + 2], base = tab[4 * i + 3];
    const long long len = (e - a) * k;
    const S* from = src + (base + a - s) * k;
    const long long o = a * k;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < len; t += (long long)gridDim.x * blockDim.x) {
        const S v = from[t];
        if (dst) dst[o + t] = v;
        if (MODE == OUT_SET64) x64[o + t] = (double)v;
        if (MODE == OUT_ADD64) x64[o + t] += (double)v;
    }
}

dim3 part_grid(const PartPlan* q, int k)
{
    const long long per_block = (long long)q->n_ext * k / std::max(1, q->P);
    long long bx = (per_block + 4 * 256 - 1) / (4 * 256);
    bx = std::max<long long>(1, std::min<long long>(bx, std::max(1, 4096 / q->P)));
    return dim3((unsigned)bx, (unsigned)q->P);
}

}  // namespace

int download_natural_csr(sptrsv_plan_s* p, std::vector<int>& rp, std::vector<int>& ci, std::vector<double>& va)
{
    HostCsr h;
    int e = download_natural(p, h);
    if (e) return e;
    rp.swap(h.rp);
    ci.swap(h.ci);
    va.swap(h.va);
    return 0;
}

static void part_delete(PartPlan* q)
{
    if (!q) return;
    if (q->sub) sptrsv_plan_destroy(q->sub);
    if (q->info.row_ctr || q->ext.ia) free_device_analysis(&q->ext, &q->info);
    cudaFree(q->d_tab);
    cudaFree(q->bx); cudaFree(q->xx); cudaFree(q->bx32); cudaFree(q->xx32);
    delete q;
}

void part_free(sptrsv_plan_s* p)
{
    part_delete(p->part);
    part_delete(p->part_alt);
    p->part = p->part_alt = nullptr;
}

// Blocks of a host CSR (natural order, diagonal last): P block starts near
// i n / P at run starts, and each block's warm-up start.  tab gets 4 ints per
// block (s, a, e, 0); *reach, *bound as in PartPlan.  threads: host threads
// for the per-block searches (1: the caller's thread only).  min_ratio > 0:
// the warm-up is first measured on a probe block in the middle of the
// matrix, and P is lowered so that blocks hold at least min_ratio times it
// (SPTRSV_ERR_UNSUPPORTED when fewer than 2 blocks remain).
int partition_blocks(const int* rp, const int* ci, const double* va, int n, int P, int threads,
                     std::vector<int>& tab, int* reach, double* bound, double min_ratio)
{
    if (P < 2 || P > 4096) return set_error(SPTRSV_ERR_INVALID_ARG, "partitions: P must be in [2, 4096]");
    if ((long long)n < 64LL * P)
        return set_error(SPTRSV_ERR_UNSUPPORTED, "partitions: %d rows are too few for %d blocks", n, P);
    HostCsr L;
    L.n = n;
    L.rp.assign(rp, rp + n + 1);
    L.ci.assign(ci, ci + rp[n]);
    L.va.assign(va, va + rp[n]);
    // reach, most off-diagonals per row, diagonal dominance, run starts
    int w = 1, maxoff = 0;
    std::vector<unsigned char> run0(n, 1);
    for (int r = 0; r < n; r++) {
        const int p0 = L.rp[r], p1 = L.rp[r + 1] - 1;
        maxoff = std::max(maxoff, p1 - p0);
        double off = 0;
        for (int t = p0; t < p1; t++) {
            off += std::fabs(L.va[t]);
            w = std::max(w, r - L.ci[t]);
            if (L.ci[t] == r - 1) run0[r] = 0;
        }
        if (!(std::fabs(L.va[p1]) >= off))
            return set_error(SPTRSV_ERR_UNSUPPORTED, "partitions: row %d is not diagonally dominant "
                             "(|L_ii| < sum |L_ij|); a partitioned solve needs every row to be", r);
    }
    // the bound costs a dense row of the spike per row: used when that is cheap
    const bool spike = (long long)std::min(w, n) * std::max(1, maxoff) <= kSpikeMaxWork;
    int Kprobe = 0;
    if (min_ratio > 0) {
        const int ap = run_start_below(run0, n / 2, w);
        double bp = 0;
        const int sp = find_start(L, run0, ap, std::min(n, ap + n / P), w, maxoff, spike, 2 * w, &bp);
        Kprobe = ap - sp;
        const long long Pmax = (long long)(n / (min_ratio * std::max(1, Kprobe)));
        if (Pmax < P) P = (int)Pmax;
        if (P < 2)
            return set_error(SPTRSV_ERR_UNSUPPORTED, "partitions: a warm-up of %d rows leaves no room for 2 blocks",
                             Kprobe);
    }
    // block starts: run starts near i n / P
    std::vector<int> a(P + 1);
    a[0] = 0;
    a[P] = n;
    for (int i = 1; i < P; i++) {
        const int t = (int)((long long)i * n / P);
        int best = t;
        for (int d = 0; d <= w / 2; d++) {
            if (t - d > a[i - 1] && run0[t - d]) {
                best = t - d;
                break;
            }
            if (t + d < n && run0[t + d]) {
                best = t + d;
                break;
            }
        }
        a[i] = std::max(best, a[i - 1] + 1);
    }
    for (int i = 1; i <= P; i++)
        if (a[i] <= a[i - 1]) return set_error(SPTRSV_ERR_UNSUPPORTED, "partitions: empty block");
    // warm-up starts: block 1 searched from scratch (or from the probe), the
    // rest from its result, in parallel
    std::vector<int> s(P, 0);
    std::vector<double> bnd(P, 0.0);
    s[1] = find_start(L, run0, a[1], a[2], w, maxoff, spike, Kprobe > 0 ? Kprobe : 2 * w, &bnd[1], Kprobe == 0);
    const int K1 = std::max(a[1] - s[1], Kprobe);
    {
        const int nt = std::max(1, std::min<int>(P - 2, threads));
        std::vector<std::thread> th;
        auto work = [&](int t) {
            for (int i = 2 + t; i < P; i += nt)
                s[i] = find_start(L, run0, a[i], a[i + 1], w, maxoff, spike, K1, &bnd[i], false);
        };
        if (nt == 1) {
            work(0);
        } else {
            for (int t = 0; t < nt; t++) th.emplace_back(work, t);
            for (auto& x : th) x.join();
        }
    }
    tab.assign(4 * (size_t)P, 0);
    double b = 0;
    for (int i = 0; i < P; i++) {
        tab[4 * i] = s[i];
        tab[4 * i + 1] = a[i];
        tab[4 * i + 2] = a[i + 1];
        b = std::max(b, bnd[i]);
    }
    *reach = w;
    *bound = b;
    return 0;
}

int build_part(sptrsv_plan_s* p, int P)
{
    if (p->part && p->part->P == P) return 0;
    // the two most recent block systems are kept (an autotuner alternates them)
    if (p->part_alt && p->part_alt->P == P) {
        std::swap(p->part, p->part_alt);
        return 0;
    }
    // built aside; the plan's block systems change only once this one is complete
    const int n = p->n;
    if (P < 2 || P > 4096) return set_error(SPTRSV_ERR_INVALID_ARG, "partitions: P must be in [2, 4096]");
    if ((long long)n < 256LL * P)  // blocks of fewer rows would be mostly warm-up
        return set_error(SPTRSV_ERR_UNSUPPORTED, "partitions: %d rows are too few for %d blocks of >= 256 rows", n, P);
    HostCsr L;
    int e = download_natural(p, L);
    if (e) return e;
    std::vector<int> tab;
    int w = 0;
    double bound = 0;
    e = partition_blocks(L.rp.data(), L.ci.data(), L.va.data(), n, P, (int)std::thread::hardware_concurrency(), tab,
                         &w, &bound, 0.0);
    if (e) return e;
    std::vector<int> s(P), a(P + 1);
    for (int i = 0; i < P; i++) {
        s[i] = tab[4 * i];
        a[i] = tab[4 * i + 1];
    }
    a[P] = n;
    // the block system
    PartPlan* q = new PartPlan();
    q->P = P;
    q->reach = w;
    q->tab = tab;
    q->bound = bound;
    long long next = 0, nnz = 0;
    for (int i = 0; i < P; i++) {
        q->tab[4 * i + 3] = (int)next;
        next += a[i + 1] - s[i];
        q->warm_rows += a[i] - s[i];
        for (int r = s[i]; r < a[i + 1]; r++)
            for (int t = L.rp[r]; t < L.rp[r + 1]; t++) nnz += L.ci[t] >= s[i];
    }
    if (next > INT32_MAX - 1 || nnz > INT32_MAX) {
        delete q;
        return set_error(SPTRSV_ERR_UNSUPPORTED, "partitions: the block system is too large");
    }
    q->n_ext = (int)next;
    q->nnz_ext = nnz;
    std::vector<int> erp(q->n_ext + 1), eci((size_t)nnz);
    std::vector<double> eva((size_t)nnz);
    {
        long long o = 0;
        int row = 0;
        erp[0] = 0;
        for (int i = 0; i < P; i++) {
            const int si = s[i], base = q->tab[4 * i + 3];
            for (int r = si; r < a[i + 1]; r++) {
                for (int t = L.rp[r]; t < L.rp[r + 1]; t++)
                    if (L.ci[t] >= si) {
                        eci[o] = L.ci[t] - si + base;
                        eva[o] = L.va[t];
                        o++;
                    }
                erp[++row] = (int)o;
            }
        }
    }
    auto fail = [&](int code) {
        part_delete(q);
        return code;
    };
    e = allocate_memory(erp.data(), eci.data(), eva.data(), q->n_ext, &q->ext, ALL);
    if (e) return fail(e);
    q->info.mode = ALL;
    e = run_analysis_impl(&q->info, &q->ext, ALL);
    if (e) return fail(e);
    e = sptrsv_plan_create(&q->ext, &q->info, &q->sub);
    if (e) return fail(e);
    q->sub->blk_starts.resize(P);
    for (int i = 0; i < P; i++) q->sub->blk_starts[i] = q->tab[4 * i + 3];
    q->sub->part_tab = q->tab;
    if (cudaMalloc((void**)&q->d_tab, sizeof(int) * q->tab.size()) != cudaSuccess ||
        cudaMemcpy(q->d_tab, q->tab.data(), sizeof(int) * q->tab.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "partitions: block table"));
    part_delete(p->part_alt);
    p->part_alt = p->part;
    p->part = q;
    return 0;
}

int part_ensure(PartPlan* q, int k)
{
    if (k <= q->cap_rhs) return 0;
    cudaFree(q->bx); cudaFree(q->xx); cudaFree(q->bx32); cudaFree(q->xx32);
    q->bx = q->xx = nullptr;
    q->bx32 = q->xx32 = nullptr;
    q->cap_rhs = 0;
    const long long m = (long long)q->n_ext * k;
    SPT_CUDA(dalloc(&q->bx, m));
    SPT_CUDA(dalloc(&q->xx, m));
    SPT_CUDA(dalloc(&q->bx32, m));
    SPT_CUDA(dalloc(&q->xx32, m));
    q->cap_rhs = k;
    return 0;
}

int part_gather64(PartPlan* q, const double* src, double* dst, int k, cudaStream_t s)
{
    k_part_gather<double><<<part_grid(q, k), 256, 0, s>>>(q->d_tab, src, dst, k);
    SPT_CUDA(cudaGetLastError());
    return 0;
}

int part_gather32(PartPlan* q, const float* src, float* dst, int k, cudaStream_t s)
{
    k_part_gather<float><<<part_grid(q, k), 256, 0, s>>>(q->d_tab, src, dst, k);
    SPT_CUDA(cudaGetLastError());
    return 0;
}

int part_scatter64(PartPlan* q, const double* src, double* dst, int k, cudaStream_t s)
{
    k_part_scatter<double, OUT_X><<<part_grid(q, k), 256, 0, s>>>(q->d_tab, src, dst, nullptr, k);
    SPT_CUDA(cudaGetLastError());
    return 0;
}

int part_scatter32(PartPlan* q, const float* src, float* out32, double* x64, int mode, int k, cudaStream_t s)
{
    const dim3 g = part_grid(q, k);
    if (mode == OUT_SET64) k_part_scatter<float, OUT_SET64><<<g, 256, 0, s>>>(q->d_tab, src, out32, x64, k);
    else if (mode == OUT_ADD64) k_part_scatter<float, OUT_ADD64><<<g, 256, 0, s>>>(q->d_tab, src, out32, x64, k);
    else k_part_scatter<float, OUT_X><<<g, 256, 0, s>>>(q->d_tab, src, out32, x64, k);
    SPT_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace sptrsv

using namespace sptrsv;

// The blocks a partitioned plan would use, computed on the host from a host
// CSR (no GPU needed): the same search as sptrsv_plan_set_schedule with
// partitions = P.
extern "C" int sptrsv_partition_blocks_host(const struct sptrsv_host_csr_s* m, int P, int* table, double* bound)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!m || !table || m->n < 1 || !m->rowptr || !m->colidx || !m->val)
            return set_error(SPTRSV_ERR_INVALID_ARG, "partition_blocks_host: bad arguments");
        if ((long long)m->n < 256LL * P)
            return set_error(SPTRSV_ERR_UNSUPPORTED, "partitions: %d rows are too few for %d blocks of >= 256 rows", m->n,
                             P);
        int bad = -1;
        int e = sptrsv_check_csr_host(m->rowptr, m->colidx, m->n, &bad);
        if (e) return e;
        std::vector<int> tab;
        int w = 0;
        double b = 0;
        e = partition_blocks(m->rowptr, m->colidx, m->val, m->n, P, (int)std::thread::hardware_concurrency(), tab, &w,
                             &b, 0.0);
        if (e) return e;
        long long next = 0;
        for (int i = 0; i < P; i++) {
            tab[4 * i + 3] = (int)next;
            next += tab[4 * i + 2] - tab[4 * i];
        }
        std::copy(tab.begin(), tab.end(), table);
        if (bound) *bound = b;
        return ok();
    });
}

extern "C" int sptrsv_plan_partition_info(sptrsv_plan_t p, int* blocks, int* n_ext, long long* warm_rows,
                                          double* bound, int* table)
{
    return ::sptrsv::abi_guard([&]() -> int {
        if (!p) return set_error(SPTRSV_ERR_INVALID_ARG, "partition_info: NULL plan");
        if (!p->part || p->sched.partitions < 2)
            return set_error(SPTRSV_ERR_INVALID_ARG, "partition_info: the plan's schedule is not partitioned");
        const PartPlan* q = p->part;
        if (blocks) *blocks = q->P;
        if (n_ext) *n_ext = q->n_ext;
        if (warm_rows) *warm_rows = q->warm_rows;
        if (bound) *bound = q->bound;
        if (table) std::copy(q->tab.begin(), q->tab.end(), table);
        return ok();
    });
}
