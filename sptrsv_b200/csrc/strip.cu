// strip.cu — the STRIP schedule: natural-order chunks solved by a prefix scan.
//
// Rows are cut into chunks of consecutive rows (natural order): a chunk
// starts at every row that does not depend on the row before it (a grid
// line's first cell) and after 32 rows.  The schedule applies when every
// dependency of a row that falls inside its own chunk is on the row just
// before it (the lower triangles of 2D and 3D stencils in natural order: the
// left neighbour is inside the chunk, the neighbours above and behind are
// outside).  A chunk is then solved by one warp, lane j owning row j:
//   alpha_j = (b_j - sum of the entries outside the chunk) / L_jj,
//   beta_j  = -L_j,j-1 / L_jj   (0 for the first row of the chunk),
//   x_j     = alpha_j + beta_j x_{j-1},
// a first-order linear recurrence evaluated by a 5-step affine prefix scan
// (Kogge-Stone over the warp) instead of 32 dependent steps.
//
// A run is a maximal sequence of chunks each of whose first row depends on
// the last row of the chunk before: with the cut above, a grid line of any
// length.  R consecutive runs form a strip, solved by one warp in wavefront
// order: chunk k of every run of the strip, then chunk k + 1, so the
// dependency on the previous line is, for all but the strip's first run, a
// chunk this warp solved a moment ago.  When that order would put a
// dependency after its user, the strip's chunks are taken in the order of
// their level in the chunk dependency graph instead, which is topological
// for any matrix.  The last W = 2R chunks a
// warp solved stay in a shared-memory ring; entries that point there are
// encoded as ~slot, the rest are read from x with the usual value-as-flag
// wait.  Strips are in natural order and every dependency points to an
// earlier strip or to an earlier position in the same strip, so persistent
// warps taking strips round-robin cannot deadlock.
//
// The layout is stored in processing order (slot = position * 32 + lane), so
// the kernel can load a chunk's metadata two chunks ahead and its entries one
// chunk ahead without a dependent load.
#include <algorithm>
#include <vector>

#include "internal.h"
#include "plan.h"

namespace sptrsv {

namespace {

// brk[i] = 1 when row i does not depend on row i - 1 (a chunk starts there).
__global__ void k_strip_breaks(SptLayout l, const int* __restrict__ inv, int n, unsigned char* __restrict__ brk)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = inv[i];
        const int s = l.ptr[p], e = l.ptr[p + 1];
        brk[i] = (unsigned char)(i == 0 || e == s || l.col[e - 1] != i - 1);  // columns ascend: the last is largest
    }
}

// Per natural row: entries before its chunk (a sorted prefix) and the value
// of the one allowed entry inside the chunk (column i-1).  flag |= 1 when a
// row has any other entry inside its chunk.
__global__ void k_strip_rows(SptLayout l, const int* __restrict__ inv, int n, const int* __restrict__ rchunk,
                             const int* __restrict__ cstart, int* __restrict__ ecnt, double* __restrict__ lsub64,
                             double* __restrict__ di64, float* __restrict__ di32, int* __restrict__ flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int cs = cstart[rchunk[i]];
        const int p = inv[i];
        const int s = l.ptr[p], e = l.ptr[p + 1];
        int ext = 0, bad = 0;
        double lv = 0.0;
        for (int t = s; t < e; t++) {
            const int c = l.col[t];
            if (c >= cs) {
                if (c != i - 1) bad = 1;
                else lv = l.val64[t];
            } else {
                ext++;
            }
        }
        ecnt[i] = ext;
        lsub64[i] = lv;
        di64[i] = l.di64[p];
        di32[i] = l.di32[p];
        if (bad) atomicOr(flag, 1);
    }
}

// The natural column of every entry before its row's chunk, in eptr order.
__global__ void k_strip_extcols(SptLayout l, const int* __restrict__ inv, int n, const int* __restrict__ eptr,
                                int* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = l.ptr[inv[i]], o = eptr[i], cnt = eptr[i + 1] - o;
        for (int t = 0; t < cnt; t++) out[o + t] = l.col[s + t];
    }
}

// Slot metadata in processing order; cnt[slot] = entries of the slot's row.
__global__ void k_strip_slots(const int* __restrict__ chunk_at, const int* __restrict__ cstart, int nslots,
                              const int* __restrict__ eptr, const double* __restrict__ nlsub,
                              const double* __restrict__ ndi, const float* __restrict__ ndi32, int* __restrict__ row,
                              int* __restrict__ cnt, double* __restrict__ lsub64, float* __restrict__ lsub32,
                              double* __restrict__ di64, float* __restrict__ di32)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nslots; t += gridDim.x * blockDim.x) {
        const int q = chunk_at[t >> 5];
        const int i = cstart[q] + (t & 31);
        const bool own = i < cstart[q + 1];
        row[t] = own ? i : -1;
        cnt[t] = own ? eptr[i + 1] - eptr[i] : 0;
        lsub64[t] = own ? nlsub[i] : 0.0;
        lsub32[t] = own ? (float)nlsub[i] : 0.0f;
        di64[t] = own ? ndi[i] : 0.0;
        di32[t] = own ? ndi32[i] : 0.0f;
    }
}

// *out = max(*out, a[0..n)) (non-negative values).
__global__ void k_max_int(const int* __restrict__ a, int n, int* out)
{
    int m = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) m = max(m, a[t]);
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, m);
}

// Entries in processing order, encoded: ~slot for a column whose chunk this
// warp solved fewer than W positions earlier in the same strip, else the
// column.  flag |= 2 when a same-strip dependency does not come earlier.
__global__ void k_strip_fill(SptLayout l, const int* __restrict__ inv, const int* __restrict__ row, int nslots,
                             const int* __restrict__ rchunk, const int* __restrict__ cstart,
                             const int* __restrict__ pe, const int* __restrict__ strip_of,
                             const int* __restrict__ pos_of, int W, int* __restrict__ ecol,
                             double* __restrict__ ev64, float* __restrict__ ev32, int* __restrict__ flag)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nslots; t += gridDim.x * blockDim.x) {
        const int i = row[t];
        if (i < 0) continue;
        const int q = rchunk[i], sq = strip_of[q], pq = pos_of[q];
        const int s = l.ptr[inv[i]];
        const int o = pe[t], cnt = pe[t + 1] - o;
        for (int k = 0; k < cnt; k++) {
            const int c = l.col[s + k];
            const int qc = rchunk[c];
            int enc = c;
            if (strip_of[qc] == sq) {
                const int d = pq - pos_of[qc];
                if (d <= 0) atomicOr(flag, 2);
                else if (d < W) enc = ~((pos_of[qc] % W) * 32 + (c - cstart[qc]));
            }
            ecol[o + k] = enc;
            ev64[o + k] = l.val64[s + k];
            ev32[o + k] = l.val32[s + k];
        }
    }
}

// WAVE entries (natural chunk order): a column inside the row's group is
// encoded as ~(column - first row of the group), its value is then read
// from the CTA's shared-memory copy.
__global__ void k_wave_fill(SptLayout l, const int* __restrict__ inv, const int* __restrict__ row, int nslots,
                            const int* __restrict__ rchunk, const int* __restrict__ chunk_g0,
                            const int* __restrict__ pe, int* __restrict__ ecol, double* __restrict__ ev64,
                            float* __restrict__ ev32)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nslots; t += gridDim.x * blockDim.x) {
        const int i = row[t];
        if (i < 0) continue;
        const int g0 = chunk_g0[rchunk[i]];
        const int s = l.ptr[inv[i]];
        const int o = pe[t], cnt = pe[t + 1] - o;
        for (int k = 0; k < cnt; k++) {
            const int c = l.col[s + k];
            ecol[o + k] = c >= g0 ? ~(c - g0) : c;
            ev64[o + k] = l.val64[s + k];
            ev32[o + k] = l.val32[s + k];
        }
    }
}

}  // namespace

void strip_free(StripLayout& t)
{
    cudaFree(t.row); cudaFree(t.pe); cudaFree(t.ecol); cudaFree(t.ev64); cudaFree(t.ev32); cudaFree(t.lsub64);
    cudaFree(t.lsub32); cudaFree(t.di64); cudaFree(t.di32); cudaFree(t.sptr);
    t = StripLayout{};
}

void wave_free(WaveLayout& w)
{
    cudaFree(w.row); cudaFree(w.pe); cudaFree(w.ecol); cudaFree(w.ev64); cudaFree(w.ev32); cudaFree(w.lsub64);
    cudaFree(w.lsub32); cudaFree(w.di64); cudaFree(w.di32); cudaFree(w.runc); cudaFree(w.grun); cudaFree(w.grow);
    cudaFree(w.gseq); cudaFree(w.brow); cudaFree(w.ghx);
    w = WaveLayout{};
}

namespace {

// The chunk cut and the per-row data both layouts start from.
struct Chunks {
    std::vector<int> cstart, rchunk;   // host: first row of each chunk (+ n), chunk of each row
    std::vector<unsigned char> linked; // host: chunk continues the previous chunk's run
    int nch = 0, m = 0;                // chunks, entries before their rows' chunks
    int *d_rchunk = nullptr, *d_cstart = nullptr, *eptr = nullptr;
    double *nlsub = nullptr, *ndi = nullptr;
    float* ndi32 = nullptr;
    void release()
    {
        cudaFree(d_rchunk); cudaFree(d_cstart); cudaFree(eptr); cudaFree(nlsub); cudaFree(ndi); cudaFree(ndi32);
        d_rchunk = d_cstart = eptr = nullptr;
        nlsub = ndi = nullptr;
        ndi32 = nullptr;
    }
};

// Cuts the chunks, checks the structure (SPTRSV_ERR_UNSUPPORTED otherwise)
// and fills the per-natural-row arrays.  On error everything is released.
int chunk_analysis(sptrsv_plan_s* p, Chunks& c, cudaStream_t s)
{
    const int n = p->n;
    unsigned char* brk = nullptr;
    int *ecnt = nullptr, *flag = nullptr, *scr = nullptr;
    auto cleanup = [&]() {
        cudaFree(brk); cudaFree(ecnt); cudaFree(flag); cudaFree(scr);
    };
    auto fail = [&](int code) {
        cleanup();
        c.release();
        return code;
    };
#define CCHK(call)                                                \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, #call)); \
    } while (0)
    // chunks: a new one at every row that does not depend on the row before
    // it, and after 32 rows
    CCHK(dalloc(&brk, n));
    k_strip_breaks<<<grid_for(n, 256), 256, 0, s>>>(p->lev, p->inv, n, brk);
    CCHK(cudaGetLastError());
    std::vector<unsigned char> hbrk(n);
    CCHK(cudaMemcpy(hbrk.data(), brk, (size_t)n, cudaMemcpyDeviceToHost));
    c.cstart.clear();
    c.linked.clear();
    c.rchunk.assign(n, 0);
    for (int i = 0; i < n; i++) {
        if (hbrk[i] || i - c.cstart.back() == 32) {
            c.cstart.push_back(i);
            c.linked.push_back((unsigned char)!hbrk[i]);
        }
        c.rchunk[i] = (int)c.cstart.size() - 1;
    }
    c.nch = (int)c.cstart.size();
    c.cstart.push_back(n);
    CCHK(dalloc(&c.d_rchunk, n));
    CCHK(dalloc(&c.d_cstart, c.nch + 1));
    CCHK(cudaMemcpy(c.d_rchunk, c.rchunk.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    CCHK(cudaMemcpy(c.d_cstart, c.cstart.data(), sizeof(int) * ((size_t)c.nch + 1), cudaMemcpyHostToDevice));
    // per natural row: entries before the chunk, L(i, i-1), 1/diagonal
    CCHK(dalloc(&ecnt, (long long)n + 1));
    CCHK(dalloc(&flag, 1));
    CCHK(dalloc(&c.nlsub, n));
    CCHK(dalloc(&c.ndi, n));
    CCHK(dalloc(&c.ndi32, n));
    CCHK(cudaMemsetAsync(flag, 0, sizeof(int), s));
    CCHK(cudaMemsetAsync(ecnt + n, 0, sizeof(int), s));
    k_strip_rows<<<grid_for(n, 256), 256, 0, s>>>(p->lev, p->inv, n, c.d_rchunk, c.d_cstart, ecnt, c.nlsub, c.ndi,
                                                  c.ndi32, flag);
    CCHK(cudaGetLastError());
    int hflag = 0;
    CCHK(cudaMemcpy(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (hflag) return fail(set_error(SPTRSV_ERR_UNSUPPORTED, "strip schedule: a row depends on a row of its own "
                                                              "chunk other than the one before it"));
    CCHK(dalloc(&c.eptr, (long long)n + 1));
    CCHK(dalloc(&scr, scan_scratch_ints((long long)n + 1)));
    CCHK(scan_exclusive(ecnt, c.eptr, (long long)n + 1, scr, s));
    CCHK(cudaMemcpy(&c.m, c.eptr + n, sizeof(int), cudaMemcpyDeviceToHost));
#undef CCHK
    cleanup();
    return 0;
}

}  // namespace

int build_strip_layout(sptrsv_plan_s* p, int R)
{
    if (p->row_strip_R == R && p->strip.row) return 0;
    strip_free(p->strip);
    p->row_strip_R = 0;
    const int n = p->n;
    const int W = 2 * R;
    cudaStream_t s = 0;
    StripLayout t{};
    Chunks ch;
    {
        int e = chunk_analysis(p, ch, s);
        if (e) return e;
    }
    const int nch = ch.nch, nslots = nch * 32, m = ch.m;
    const std::vector<int>& cstart = ch.cstart;
    const std::vector<int>& rchunk = ch.rchunk;
    const std::vector<unsigned char>& linked = ch.linked;
    int *ext = nullptr, *flag = nullptr, *scr = nullptr, *d_strip_of = nullptr, *d_pos = nullptr,
        *d_chunk_at = nullptr, *scnt = nullptr;
    int* eptr = ch.eptr;
    auto cleanup = [&]() {
        cudaFree(ext); cudaFree(flag); cudaFree(scr); cudaFree(d_strip_of); cudaFree(d_pos); cudaFree(d_chunk_at);
        cudaFree(scnt);
        ch.release();
    };
    auto fail = [&](int code) {
        cleanup();
        strip_free(t);
        return code;
    };
#define SCHK(call)                                                \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, #call)); \
    } while (0)
    SCHK(dalloc(&flag, 1));
    SCHK(cudaMemsetAsync(flag, 0, sizeof(int), s));
    SCHK(dalloc(&scr, scan_scratch_ints((long long)nslots + 1)));
    // 3. their columns on the host: chunk dependencies
    SCHK(dalloc(&ext, m));
    k_strip_extcols<<<grid_for(n, 256), 256, 0, s>>>(p->lev, p->inv, n, eptr, ext);
    SCHK(cudaGetLastError());
    std::vector<int> heptr((size_t)n + 1), hcol((size_t)m);
    SCHK(cudaMemcpy(heptr.data(), eptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost));
    SCHK(cudaMemcpy(hcol.data(), ext, sizeof(int) * (size_t)m, cudaMemcpyDeviceToHost));
    // 4. runs and strips; wavefront order (chunk k of each run) when it is
    //    topological, else chunk-level order
    std::vector<int> run0;
    for (int q = 0; q < nch; q++)
        if (q == 0 || !linked[q]) run0.push_back(q);
    const int nruns = (int)run0.size();
    run0.push_back(nch);
    const int nstrips = (nruns + R - 1) / R;
    std::vector<int> sptr(nstrips + 1, 0), order(nch), strip_of(nch), pos_of(nch);
    auto deps_ok = [&](int q) {  // every same-strip dependency of chunk q comes earlier
        for (int e = heptr[cstart[q]]; e < heptr[cstart[q + 1]]; e++) {
            const int qc = rchunk[hcol[e]];
            if (strip_of[qc] == strip_of[q] && pos_of[qc] >= pos_of[q]) return false;
        }
        return true;
    };
    std::vector<int> clev;
    for (int st = 0; st < nstrips; st++) {
        const int r0 = st * R, r1 = std::min(nruns, r0 + R);
        const int q0 = run0[r0], q1 = run0[r1];
        sptr[st + 1] = q1;
        int maxlen = 0, k = q0;
        for (int r = r0; r < r1; r++) maxlen = std::max(maxlen, run0[r + 1] - run0[r]);
        for (int j = 0; j < maxlen; j++)
            for (int r = r0; r < r1; r++)
                if (j < run0[r + 1] - run0[r]) order[k++] = run0[r] + j;
        for (int t2 = q0; t2 < q1; t2++) {
            strip_of[order[t2]] = st;
            pos_of[order[t2]] = t2 - q0;
        }
        bool ok = true;
        for (int q = q0; q < q1 && ok; q++) ok = deps_ok(q);
        if (!ok) {
            if (clev.empty()) {  // chunk levels: 1 + the largest level among the chunks a chunk reads
                clev.assign(nch, 0);
                for (int q = 0; q < nch; q++) {
                    int lv = 0;
                    for (int e = heptr[cstart[q]]; e < heptr[cstart[q + 1]]; e++)
                        lv = std::max(lv, clev[rchunk[hcol[e]]]);
                    clev[q] = lv + 1;
                }
            }
            for (int q = q0; q < q1; q++) order[q] = q;
            std::stable_sort(order.begin() + q0, order.begin() + q1,
                             [&](int a, int b) { return clev[a] < clev[b]; });
            for (int t2 = q0; t2 < q1; t2++) pos_of[order[t2]] = t2 - q0;
        }
    }
    SCHK(dalloc(&t.sptr, nstrips + 1));
    SCHK(dalloc(&d_chunk_at, nch));
    SCHK(dalloc(&d_strip_of, nch));
    SCHK(dalloc(&d_pos, nch));
    SCHK(cudaMemcpy(t.sptr, sptr.data(), sizeof(int) * sptr.size(), cudaMemcpyHostToDevice));
    SCHK(cudaMemcpy(d_chunk_at, order.data(), sizeof(int) * (size_t)nch, cudaMemcpyHostToDevice));
    SCHK(cudaMemcpy(d_strip_of, strip_of.data(), sizeof(int) * (size_t)nch, cudaMemcpyHostToDevice));
    SCHK(cudaMemcpy(d_pos, pos_of.data(), sizeof(int) * (size_t)nch, cudaMemcpyHostToDevice));
    // 5. slots and entries in processing order
    SCHK(dalloc(&t.row, nslots));
    SCHK(dalloc(&scnt, (long long)nslots + 1));
    SCHK(dalloc(&t.lsub64, nslots));
    SCHK(dalloc(&t.lsub32, nslots));
    SCHK(dalloc(&t.di64, nslots));
    SCHK(dalloc(&t.di32, nslots));
    SCHK(cudaMemsetAsync(scnt + nslots, 0, sizeof(int), s));
    k_strip_slots<<<grid_for(nslots, 256), 256, 0, s>>>(d_chunk_at, ch.d_cstart, nslots, eptr, ch.nlsub, ch.ndi,
                                                        ch.ndi32, t.row, scnt, t.lsub64, t.lsub32, t.di64, t.di32);
    SCHK(cudaGetLastError());
    SCHK(dalloc(&t.pe, (long long)nslots + 1));
    SCHK(scan_exclusive(scnt, t.pe, (long long)nslots + 1, scr, s));
    SCHK(dalloc(&t.ecol, m));
    SCHK(dalloc(&t.ev64, m));
    SCHK(dalloc(&t.ev32, m));
    k_strip_fill<<<grid_for(nslots, 256), 256, 0, s>>>(p->lev, p->inv, t.row, nslots, ch.d_rchunk, ch.d_cstart, t.pe,
                                                       d_strip_of, d_pos, W, t.ecol, t.ev64, t.ev32, flag);
    SCHK(cudaGetLastError());
    int hflag = 0;
    SCHK(cudaMemcpy(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (hflag) return fail(set_error(SPTRSV_ERR_UNSUPPORTED, "strip schedule: a dependency inside a strip does not "
                                                              "come earlier in its wavefront order"));
#undef SCHK
    t.nstrips = nstrips;
    t.R = R;
    t.W = W;
    cleanup();
    p->strip = t;
    p->row_strip_R = R;
    return 0;
}

int build_wave_layout(sptrsv_plan_s* p, int G, int max_rows)
{
    if (p->wave.row && p->wave.G == G) return 0;
    wave_free(p->wave);
    cudaStream_t s = 0;
    WaveLayout w{};
    Chunks ch;
    {
        int e = chunk_analysis(p, ch, s);
        if (e) return e;
    }
    const int nch = ch.nch, nslots = nch * 32, m = ch.m;
    int *d_ident = nullptr, *d_g0 = nullptr, *scnt = nullptr, *scr = nullptr;
    auto cleanup = [&]() {
        cudaFree(d_ident); cudaFree(d_g0); cudaFree(scnt); cudaFree(scr);
        ch.release();
    };
    auto fail = [&](int code) {
        cleanup();
        wave_free(w);
        return code;
    };
#define WCHK(call)                                                \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, #call)); \
    } while (0)
    // runs (grid lines) and groups of G runs; on a block system (blk_starts
    // set) a group also ends before a run that starts a block
    std::vector<int> run0;
    for (int q = 0; q < nch; q++)
        if (q == 0 || !ch.linked[q]) run0.push_back(q);
    const int nruns = (int)run0.size();
    run0.push_back(nch);
    std::vector<int> grun, blk_of_group;
    {
        size_t nb = 0;  // blocks whose start is at or before the current run
        int in_group = 0;
        for (int r = 0; r < nruns; r++) {
            const int row = ch.cstart[run0[r]];
            bool starts_block = false;
            while (nb < p->blk_starts.size() && p->blk_starts[nb] <= row) {
                starts_block = p->blk_starts[nb] == row;
                nb++;
            }
            if (r == 0 || in_group == G || starts_block) {
                grun.push_back(r);
                blk_of_group.push_back(nb > 0 ? (int)nb - 1 : 0);
                in_group = 0;
            }
            in_group++;
        }
        grun.push_back(nruns);
    }
    const int ngroups = (int)grun.size() - 1;
    std::vector<int> grow(ngroups + 1), g0(nch), ident(nch);
    int cap = 0;
    for (int g = 0; g <= ngroups; g++) {
        grow[g] = ch.cstart[run0[grun[g]]];
        if (g > 0) cap = std::max(cap, grow[g] - grow[g - 1]);
    }
    // processing order: natural, or on a block system the blocks' groups
    // interleaved (the j-th group of every block, then the (j+1)-th), which is
    // topological because a group depends only on groups of its own block
    std::vector<int> gseq;
    if (!p->blk_starts.empty() && ngroups > 0) {
        std::vector<int> rank(ngroups);
        for (int g = 0; g < ngroups; g++)
            rank[g] = (g > 0 && blk_of_group[g] == blk_of_group[g - 1]) ? rank[g - 1] + 1 : 0;
        gseq.resize(ngroups);
        for (int g = 0; g < ngroups; g++) gseq[g] = g;
        std::stable_sort(gseq.begin(), gseq.end(), [&](int a, int b) { return rank[a] < rank[b]; });
    }
    if (cap > max_rows)
        return fail(set_error(SPTRSV_ERR_UNSUPPORTED, "wave schedule: %d lines of the matrix hold %d rows, more than "
                                                      "the %d that fit shared memory", G, cap, max_rows));
    for (int g = 0; g < ngroups; g++)
        for (int q = run0[grun[g]]; q < run0[grun[g + 1]]; q++) g0[q] = grow[g];
    for (int q = 0; q < nch; q++) ident[q] = q;
    WCHK(dalloc(&w.runc, nruns + 1));
    WCHK(dalloc(&w.grun, ngroups + 1));
    WCHK(dalloc(&w.grow, ngroups + 1));
    WCHK(dalloc(&d_ident, nch));
    WCHK(dalloc(&d_g0, nch));
    WCHK(cudaMemcpy(w.runc, run0.data(), sizeof(int) * (size_t)(nruns + 1), cudaMemcpyHostToDevice));
    WCHK(cudaMemcpy(w.grun, grun.data(), sizeof(int) * (size_t)(ngroups + 1), cudaMemcpyHostToDevice));
    WCHK(cudaMemcpy(w.grow, grow.data(), sizeof(int) * (size_t)(ngroups + 1), cudaMemcpyHostToDevice));
    if (!gseq.empty()) {
        WCHK(dalloc(&w.gseq, ngroups));
        WCHK(cudaMemcpy(w.gseq, gseq.data(), sizeof(int) * (size_t)ngroups, cudaMemcpyHostToDevice));
    }
    WCHK(cudaMemcpy(d_ident, ident.data(), sizeof(int) * (size_t)nch, cudaMemcpyHostToDevice));
    WCHK(cudaMemcpy(d_g0, g0.data(), sizeof(int) * (size_t)nch, cudaMemcpyHostToDevice));
    // slots and entries in natural chunk order
    WCHK(dalloc(&w.row, nslots));
    WCHK(dalloc(&scnt, (long long)nslots + 1));
    WCHK(dalloc(&w.lsub64, nslots));
    WCHK(dalloc(&w.lsub32, nslots));
    WCHK(dalloc(&w.di64, nslots));
    WCHK(dalloc(&w.di32, nslots));
    WCHK(cudaMemsetAsync(scnt + nslots, 0, sizeof(int), s));
    k_strip_slots<<<grid_for(nslots, 256), 256, 0, s>>>(d_ident, ch.d_cstart, nslots, ch.eptr, ch.nlsub, ch.ndi,
                                                        ch.ndi32, w.row, scnt, w.lsub64, w.lsub32, w.di64, w.di32);
    WCHK(cudaGetLastError());
    WCHK(dalloc(&scr, scan_scratch_ints((long long)nslots + 1)));
    WCHK(dalloc(&w.pe, (long long)nslots + 1));
    WCHK(scan_exclusive(scnt, w.pe, (long long)nslots + 1, scr, s));
    k_max_int<<<grid_for(nslots, 256), 256, 0, s>>>(scnt, nslots, scnt + nslots);  // scnt[nslots] was 0
    WCHK(cudaGetLastError());
    WCHK(cudaMemcpyAsync(&w.maxe, scnt + nslots, sizeof(int), cudaMemcpyDeviceToHost, s));
    WCHK(dalloc(&w.ecol, m));
    WCHK(dalloc(&w.ev64, m));
    WCHK(dalloc(&w.ev32, m));
    k_wave_fill<<<grid_for(nslots, 256), 256, 0, s>>>(p->lev, p->inv, w.row, nslots, ch.d_rchunk, d_g0, w.pe, w.ecol,
                                                      w.ev64, w.ev32);
    WCHK(cudaGetLastError());
    WCHK(cudaStreamSynchronize(s));
    if (!p->part_tab.empty() && ngroups > 0) {
        // a block system: b rows and x destinations in the outer plan's rows,
        // for its streamed host solves
        const int P = (int)p->part_tab.size() / 4;
        auto blk = [&](int row) {  // block holding a block-system row
            int lo = 0, hi = P - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (p->part_tab[4 * mid + 3] <= row) lo = mid;
                else hi = mid - 1;
            }
            return lo;
        };
        std::vector<int> hrow(nslots), hbrow(nslots, -1), hghx(2 * (size_t)ngroups);
        WCHK(cudaMemcpy(hrow.data(), w.row, sizeof(int) * (size_t)nslots, cudaMemcpyDeviceToHost));
        for (int q = 0; q < nslots; q++)
            if (hrow[q] >= 0) {
                const int b = blk(hrow[q]);
                hbrow[q] = p->part_tab[4 * b] + (hrow[q] - p->part_tab[4 * b + 3]);
            }
        for (int g = 0; g < ngroups; g++) {
            const int b = blk(grow[g]);
            const int sb = p->part_tab[4 * b], ab = p->part_tab[4 * b + 1], base = p->part_tab[4 * b + 3];
            const int nr = grow[g + 1] - grow[g];
            hghx[2 * g] = sb + (grow[g] - base);
            hghx[2 * g + 1] = std::max(0, std::min(nr, base + (ab - sb) - grow[g]));
        }
        WCHK(dalloc(&w.brow, nslots));
        WCHK(dalloc(&w.ghx, 2LL * ngroups));
        WCHK(cudaMemcpy(w.brow, hbrow.data(), sizeof(int) * (size_t)nslots, cudaMemcpyHostToDevice));
        WCHK(cudaMemcpy(w.ghx, hghx.data(), sizeof(int) * 2 * (size_t)ngroups, cudaMemcpyHostToDevice));
    }
#undef WCHK
    w.ngroups = ngroups;
    w.G = G;
    w.cap = cap;
    cleanup();
    p->wave = w;
    return 0;
}

}  // namespace sptrsv
