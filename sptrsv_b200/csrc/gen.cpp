// gen.cpp — seeded synthetic lower-triangular matrices (benchmark inputs).
//
// The reference reads SuiteSparse .mtx files (main.cu:66-246); none ship with
// it, so the benchmark configurations are generated here instead.  Every
// matrix is square lower-triangular CSR with sorted columns and the
// diagonal last (the layout main.cu:224-240 produces).  Randomness:
// xoshiro256** seeded through splitmix64; rows are generated in order from
// one stream, so a (generator, sizes, seed) triple always gives the same
// matrix.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sptrsv_b200.h"

namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed)
    {
        uint64_t z = seed;
        for (int i = 0; i < 4; i++) {
            z += 0x9E3779B97F4A7C15ULL;
            uint64_t t = z;
            t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ULL;
            t = (t ^ (t >> 27)) * 0x94D049BB133111EBULL;
            s[i] = t ^ (t >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next()
    {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double u01() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    double uniform(double a, double b) { return a + (b - a) * u01(); }
    // integer in [0, m) by multiply-shift
    uint64_t below(uint64_t m) { return (uint64_t)(((unsigned __int128)next() * m) >> 64); }
    double normal()
    {
        double u1 = u01(), u2 = u01();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// Distinct sample of k integers from [lo, hi) (Floyd's algorithm) with a
// stamped open-addressing set; returns them sorted ascending.
struct DistinctSampler {
    std::vector<int> key;
    std::vector<int64_t> stamp;
    int64_t cur = 0;
    void sample(Rng& g, int lo, int hi, int k, std::vector<int>& out)
    {
        out.clear();
        int m = hi - lo;
        if (k >= m) {
            for (int v = lo; v < hi; v++) out.push_back(v);
            return;
        }
        size_t cap = 64;
        while (cap < (size_t)4 * k) cap <<= 1;
        if (key.size() < cap) {
            key.assign(cap, 0);
            stamp.assign(cap, -1);
        }
        cur++;
        size_t mask = cap - 1;
        auto insert = [&](int v) -> bool {  // true if newly inserted
            size_t h = ((uint64_t)(uint32_t)v * 0x9E3779B97F4A7C15ULL) >> 20;
            for (size_t i = h & mask;; i = (i + 1) & mask) {
                if (stamp[i] != cur) {
                    stamp[i] = cur;
                    key[i] = v;
                    return true;
                }
                if (key[i] == v) return false;
            }
        };
        for (int j = m - k; j < m; j++) {
            int t = (int)g.below((uint64_t)j + 1);
            int v = insert(lo + t) ? lo + t : (insert(lo + j), lo + j);
            out.push_back(v);
        }
        std::sort(out.begin(), out.end());
    }
};

struct Builder {
    std::vector<int> rowptr{0};
    std::vector<int> col;
    std::vector<double> val;
    // off-diagonals U(-1,1), diagonal 1 + sum |offdiag|
    void row_dominant(Rng& g, int i, const std::vector<int>& cols)
    {
        double s = 0.0;
        for (int c : cols) {
            double v = g.uniform(-1.0, 1.0);
            col.push_back(c);
            val.push_back(v);
            s += std::fabs(v);
        }
        col.push_back(i);
        val.push_back(1.0 + s);
        rowptr.push_back((int)col.size());
    }
    int finish(sptrsv_host_csr_t* out)
    {
        int n = (int)rowptr.size() - 1;
        out->n = n;
        out->nnz = (int)col.size();
        out->rowptr = (int*)malloc(sizeof(int) * rowptr.size());
        out->colidx = (int*)malloc(sizeof(int) * (col.size() ? col.size() : 1));
        out->val = (double*)malloc(sizeof(double) * (val.size() ? val.size() : 1));
        if (!out->rowptr || !out->colidx || !out->val) {
            sptrsv_host_csr_free(out);
            return SPTRSV_ERR_ALLOC;
        }
        memcpy(out->rowptr, rowptr.data(), sizeof(int) * rowptr.size());
        if (!col.empty()) memcpy(out->colidx, col.data(), sizeof(int) * col.size());
        if (!val.empty()) memcpy(out->val, val.data(), sizeof(double) * val.size());
        return SPTRSV_OK;
    }
};

// No C++ exception leaves the C ABI: host memory that cannot be had (a
// huge n, a corrupt size) is SPTRSV_ERR_ALLOC.
template <class F>
int host_guard(F&& f) noexcept
{
    try {
        return f();
    } catch (...) {
        return SPTRSV_ERR_ALLOC;
    }
}

}  // namespace

extern "C" {

int sptrsv_gen_banded(int n, int bandwidth, int off_min, int off_max, uint64_t seed, sptrsv_host_csr_t* out)
{
    return host_guard([&]() -> int {
        if (!out || n < 0 || bandwidth < 1 || off_min < 0 || off_max < off_min) return SPTRSV_ERR_INVALID_ARG;
        memset(out, 0, sizeof(*out));
        Rng g(seed);
        DistinctSampler ds;
        Builder b;
        b.col.reserve((size_t)n * (off_max + 1));
        b.val.reserve((size_t)n * (off_max + 1));
        std::vector<int> cols;
        for (int i = 0; i < n; i++) {
            int k = off_min == off_max ? off_min : off_min + (int)g.below((uint64_t)(off_max - off_min + 1));
            int lo = std::max(0, i - bandwidth);
            k = std::min(k, i - lo);
            ds.sample(g, lo, i, k, cols);
            b.row_dominant(g, i, cols);
        }
        return b.finish(out);
    });
}

int sptrsv_gen_grid2d(int nx, int ny, uint64_t seed, sptrsv_host_csr_t* out)
{
    return host_guard([&]() -> int {
        if (!out || nx < 1 || ny < 1 || (long long)nx * ny > 0x7fffffffLL / 3) return SPTRSV_ERR_INVALID_ARG;
        memset(out, 0, sizeof(*out));
        Rng g(seed);
        Builder b;
        long long n = (long long)nx * ny;
        b.col.reserve((size_t)n * 3);
        b.val.reserve((size_t)n * 3);
        for (int r = 0; r < ny; r++)
            for (int c = 0; c < nx; c++) {
                int i = r * nx + c;
                if (r > 0) {
                    b.col.push_back(i - nx);
                    b.val.push_back(-1.0 + g.uniform(-0.1, 0.1));
                }
                if (c > 0) {
                    b.col.push_back(i - 1);
                    b.val.push_back(-1.0 + g.uniform(-0.1, 0.1));
                }
                b.col.push_back(i);
                b.val.push_back(4.0);
                b.rowptr.push_back((int)b.col.size());
            }
        return b.finish(out);
    });
}

int sptrsv_gen_grid3d(int nx, int ny, int nz, uint64_t seed, sptrsv_host_csr_t* out)
{
    return host_guard([&]() -> int {
        if (!out || nx < 1 || ny < 1 || nz < 1 || (long long)nx * ny * nz > 0x7fffffffLL / 4) return SPTRSV_ERR_INVALID_ARG;
        memset(out, 0, sizeof(*out));
        Rng g(seed);
        Builder b;
        for (int z = 0; z < nz; z++)
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    int i = (z * ny + y) * nx + x;
                    if (z > 0) {
                        b.col.push_back(i - nx * ny);
                        b.val.push_back(-1.0 + g.uniform(-0.1, 0.1));
                    }
                    if (y > 0) {
                        b.col.push_back(i - nx);
                        b.val.push_back(-1.0 + g.uniform(-0.1, 0.1));
                    }
                    if (x > 0) {
                        b.col.push_back(i - 1);
                        b.val.push_back(-1.0 + g.uniform(-0.1, 0.1));
                    }
                    b.col.push_back(i);
                    b.val.push_back(6.0);
                    b.rowptr.push_back((int)b.col.size());
                }
        return b.finish(out);
    });
}

// Off-diagonal count per row = min(Z - 1, max_off, i) with Z ~ Zipf(s) on
// {1, 2, ...}; columns distinct, uniform over all preceding rows.
int sptrsv_gen_zipf(int n, double s, int max_off, uint64_t seed, sptrsv_host_csr_t* out)
{
    return host_guard([&]() -> int {
        if (!out || n < 0 || s <= 1.0 || max_off < 0) return SPTRSV_ERR_INVALID_ARG;
        memset(out, 0, sizeof(*out));
        // zeta(s) by a long partial sum plus the Euler-Maclaurin tail
        const int N = 1000000;
        double zeta = 0.0;
        for (int k = N; k >= 1; k--) zeta += std::pow((double)k, -s);
        zeta += std::pow((double)N, 1.0 - s) / (s - 1.0) - 0.5 * std::pow((double)N, -s);
        std::vector<double> cdf(max_off > 0 ? max_off : 1);
        double acc = 0.0;
        for (int k = 1; k <= max_off; k++) {  // P(count = k-1) = P(Z = k)
            acc += std::pow((double)k, -s) / zeta;
            cdf[k - 1] = acc;
        }
        Rng g(seed);
        DistinctSampler ds;
        Builder b;
        std::vector<int> cols;
        for (int i = 0; i < n; i++) {
            double u = g.u01();
            int cnt = max_off;
            if (max_off > 0) {
                auto it = std::lower_bound(cdf.begin(), cdf.end(), u);
                if (it != cdf.end()) cnt = (int)(it - cdf.begin());
            }
            cnt = std::min(cnt, i);
            ds.sample(g, 0, i, cnt, cols);
            b.row_dominant(g, i, cols);
        }
        return b.finish(out);
    });
}

// Block-diagonal with dense lower-triangular blocks of size `block`.
int sptrsv_gen_blockdiag(int n, int block, uint64_t seed, sptrsv_host_csr_t* out)
{
    return host_guard([&]() -> int {
        if (!out || n < 0 || block < 1) return SPTRSV_ERR_INVALID_ARG;
        memset(out, 0, sizeof(*out));
        Rng g(seed);
        Builder b;
        std::vector<int> cols;
        for (int i = 0; i < n; i++) {
            cols.clear();
            for (int c = (i / block) * block; c < i; c++) cols.push_back(c);
            b.row_dominant(g, i, cols);
        }
        return b.finish(out);
    });
}

void sptrsv_host_csr_free(sptrsv_host_csr_t* m)
{
    if (!m) return;
    free(m->rowptr);
    free(m->colidx);
    free(m->val);
    memset(m, 0, sizeof(*m));
}

// dist 0: all ones, 1: U(-1,1), 2: N(0,1)
int sptrsv_gen_vector(long long m, int dist, uint64_t seed, double* out)
{
    if (m < 0 || !out || dist < 0 || dist > 2) return SPTRSV_ERR_INVALID_ARG;
    Rng g(seed);
    for (long long i = 0; i < m; i++) out[i] = dist == 0 ? 1.0 : dist == 1 ? g.uniform(-1.0, 1.0) : g.normal();
    return SPTRSV_OK;
}

// y = L x on the host (all stored entries, row-major nrhs), FP64 in column order.
int sptrsv_host_spmv(const sptrsv_host_csr_t* m, const double* x, double* y, int nrhs)
{
    if (!m || !x || !y || nrhs < 1) return SPTRSV_ERR_INVALID_ARG;
    for (int i = 0; i < m->n; i++)
        for (int k = 0; k < nrhs; k++) {
            double s = 0.0;
            for (int p = m->rowptr[i]; p < m->rowptr[i + 1]; p++) s += m->val[p] * x[(size_t)m->colidx[p] * nrhs + k];
            y[(size_t)i * nrhs + k] = s;
        }
    return SPTRSV_OK;
}

}  // extern "C"
