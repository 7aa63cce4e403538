// mtx.cpp — MatrixMarket coordinate reader and lower-triangle extraction.
//
// The reference's driver reads a .mtx file, expands symmetric storage, builds
// CSR and keeps, per row, the entries left of the diagonal followed by the
// diagonal itself, with every value forced to 1.0 (main.cu:66-246; the value
// override at :228 and :236).  This reader follows the MatrixMarket exchange
// format as published by NIST: a banner line
//   %%MatrixMarket matrix coordinate <real|integer|pattern> <general|symmetric|skew-symmetric>
// comment lines starting with '%', a size line "rows cols entries", then one
// "i j [value]" line per entry with 1-based indices.
//
// Output: square lower-triangular CSR, sorted columns, the diagonal last in
// every row.  unit_values = 1 reproduces the reference (all values 1.0); 0
// keeps the file's values for the strict lower triangle and its diagonal
// (1.0 where the file has none).  Duplicate entries are summed.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sptrsv_b200.h"

namespace {

struct Entry {
    int r, c;
    double v;
};

int fail(const char* msg)
{
    (void)msg;
    return SPTRSV_ERR_INVALID_ARG;
}

}  // namespace

extern "C" int sptrsv_read_mtx_lower(const char* path, int unit_values, sptrsv_host_csr_t* out)
{
    if (!path || !out) return SPTRSV_ERR_INVALID_ARG;
    memset(out, 0, sizeof(*out));
    FILE* f = fopen(path, "r");
    if (!f) return fail("open");
    char line[4096];
    if (!fgets(line, sizeof(line), f)) {
        fclose(f);
        return fail("empty file");
    }
    std::string banner(line);
    for (auto& ch : banner) ch = (char)std::tolower((unsigned char)ch);
    if (banner.rfind("%%matrixmarket", 0) != 0 || banner.find("matrix") == std::string::npos ||
        banner.find("coordinate") == std::string::npos || banner.find("complex") != std::string::npos ||
        banner.find("hermitian") != std::string::npos) {
        fclose(f);
        return fail("unsupported banner");
    }
    const bool pattern = banner.find("pattern") != std::string::npos;
    const bool symmetric = banner.find("symmetric") != std::string::npos && banner.find("skew") == std::string::npos;
    const bool skew = banner.find("skew-symmetric") != std::string::npos;
    long long rows = 0, cols = 0, nent = 0;
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '%') continue;
        if (sscanf(line, "%lld %lld %lld", &rows, &cols, &nent) == 3) break;
        bool blank = true;
        for (char* p = line; *p; p++)
            if (!std::isspace((unsigned char)*p)) blank = false;
        if (!blank) {
            fclose(f);
            return fail("bad size line");
        }
    }
    if (rows <= 0 || rows != cols || rows > 0x7ffffffeLL || nent < 0) {
        fclose(f);
        return fail("matrix must be square");
    }
    const int n = (int)rows;
    std::vector<Entry> e;
    e.reserve((size_t)nent * (symmetric || skew ? 2 : 1));
    for (long long k = 0; k < nent; k++) {
        if (!fgets(line, sizeof(line), f)) {
            fclose(f);
            return fail("truncated");
        }
        if (line[0] == '%') {
            k--;
            continue;
        }
        long long i = 0, j = 0;
        double v = 1.0;
        int got = pattern ? sscanf(line, "%lld %lld", &i, &j) : sscanf(line, "%lld %lld %lf", &i, &j, &v);
        if (got < (pattern ? 2 : 3) || i < 1 || j < 1 || i > rows || j > cols) {
            fclose(f);
            return fail("bad entry");
        }
        e.push_back({(int)(i - 1), (int)(j - 1), v});
        if ((symmetric || skew) && i != j) e.push_back({(int)(j - 1), (int)(i - 1), skew ? -v : v});
    }
    fclose(f);
    // keep the lower triangle (and the diagonal), sort by (row, col), sum duplicates
    std::vector<Entry> low;
    low.reserve(e.size());
    for (const Entry& x : e)
        if (x.c <= x.r) low.push_back(x);
    std::sort(low.begin(), low.end(), [](const Entry& a, const Entry& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
    std::vector<int> rp(n + 1, 0), ci;
    std::vector<double> va;
    ci.reserve(low.size() + n);
    va.reserve(low.size() + n);
    size_t q = 0;
    for (int r = 0; r < n; r++) {
        double dval = 1.0;
        while (q < low.size() && low[q].r == r) {
            const int c = low[q].c;
            double s = 0.0;
            while (q < low.size() && low[q].r == r && low[q].c == c) s += low[q++].v;
            if (c < r) {
                ci.push_back(c);
                va.push_back(unit_values ? 1.0 : s);
            } else {
                dval = s;
            }
        }
        ci.push_back(r);  // the diagonal, last (main.cu:235-237)
        va.push_back(unit_values ? 1.0 : dval);
        rp[r + 1] = (int)ci.size();
    }
    out->n = n;
    out->nnz = (int)ci.size();
    out->rowptr = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    out->colidx = (int*)malloc(sizeof(int) * ci.size());
    out->val = (double*)malloc(sizeof(double) * va.size());
    if (!out->rowptr || !out->colidx || !out->val) {
        sptrsv_host_csr_free(out);
        return SPTRSV_ERR_ALLOC;
    }
    memcpy(out->rowptr, rp.data(), sizeof(int) * (size_t)(n + 1));
    memcpy(out->colidx, ci.data(), sizeof(int) * ci.size());
    memcpy(out->val, va.data(), sizeof(double) * va.size());
    return SPTRSV_OK;
}
