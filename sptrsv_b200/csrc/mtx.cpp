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
#include <memory>
#include <new>
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

struct FileCloser {
    void operator()(FILE* f) const
    {
        if (f) fclose(f);
    }
};

// One whole line (any length, without its newline); false at end of file.
bool read_line(FILE* f, std::string& line)
{
    line.clear();
    char buf[4096];
    while (fgets(buf, sizeof(buf), f)) {
        line += buf;
        if (!line.empty() && line.back() == '\n') {
            line.pop_back();
            return true;
        }
    }
    return !line.empty();
}

int read_mtx_lower(const char* path, int unit_values, sptrsv_host_csr_t* out)
{
    std::unique_ptr<FILE, FileCloser> f(fopen(path, "r"));
    if (!f) return fail("open");
    std::string line;
    if (!read_line(f.get(), line)) return fail("empty file");
    std::string banner(line);
    for (auto& ch : banner) ch = (char)std::tolower((unsigned char)ch);
    if (banner.rfind("%%matrixmarket", 0) != 0 || banner.find("matrix") == std::string::npos ||
        banner.find("coordinate") == std::string::npos || banner.find("complex") != std::string::npos ||
        banner.find("hermitian") != std::string::npos)
        return fail("unsupported banner");
    const bool pattern = banner.find("pattern") != std::string::npos;
    const bool symmetric = banner.find("symmetric") != std::string::npos && banner.find("skew") == std::string::npos;
    const bool skew = banner.find("skew-symmetric") != std::string::npos;
    long long rows = 0, cols = 0, nent = 0;
    while (read_line(f.get(), line)) {
        if (!line.empty() && line[0] == '%') continue;
        if (sscanf(line.c_str(), "%lld %lld %lld", &rows, &cols, &nent) == 3) break;
        for (char ch : line)
            if (!std::isspace((unsigned char)ch)) return fail("bad size line");
    }
    if (rows <= 0 || rows != cols || rows > 0x7ffffffeLL || nent < 0) return fail("matrix must be square");
    const int n = (int)rows;
    std::vector<Entry> e;
    // the size line is not trusted for memory: the vector grows with the entries actually read
    e.reserve((size_t)std::min<long long>(nent, 1LL << 22) * (symmetric || skew ? 2 : 1));
    for (long long k = 0; k < nent; k++) {
        if (!read_line(f.get(), line)) return fail("truncated");
        if (!line.empty() && line[0] == '%') {
            k--;
            continue;
        }
        long long i = 0, j = 0;
        double v = 1.0;
        int got = pattern ? sscanf(line.c_str(), "%lld %lld", &i, &j) : sscanf(line.c_str(), "%lld %lld %lf", &i, &j, &v);
        if (got < (pattern ? 2 : 3) || i < 1 || j < 1 || i > rows || j > cols) return fail("bad entry");
        e.push_back({(int)(i - 1), (int)(j - 1), v});
        if ((symmetric || skew) && i != j) e.push_back({(int)(j - 1), (int)(i - 1), skew ? -v : v});
    }
    f.reset();
    // keep the lower triangle (and the diagonal), sort by (row, col), sum duplicates
    std::vector<Entry> low;
    low.reserve(e.size());
    for (const Entry& x : e)
        if (x.c <= x.r) low.push_back(x);
    e.clear();
    e.shrink_to_fit();
    if ((long long)low.size() + n > 0x7fffffffLL) return SPTRSV_ERR_UNSUPPORTED;  // int32 row pointers
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
            double sum = 0.0;
            while (q < low.size() && low[q].r == r && low[q].c == c) sum += low[q++].v;
            if (c < r) {
                ci.push_back(c);
                va.push_back(unit_values ? 1.0 : sum);
            } else {
                dval = sum;
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

}  // namespace

// No C++ exception leaves the C ABI: running out of host memory on a large
// (or corrupt) file is SPTRSV_ERR_ALLOC.
extern "C" int sptrsv_read_mtx_lower(const char* path, int unit_values, sptrsv_host_csr_t* out)
{
    if (!path || !out) return SPTRSV_ERR_INVALID_ARG;
    memset(out, 0, sizeof(*out));
    try {
        return read_mtx_lower(path, unit_values, out);
    } catch (const std::bad_alloc&) {
        sptrsv_host_csr_free(out);
        return SPTRSV_ERR_ALLOC;
    } catch (...) {
        sptrsv_host_csr_free(out);
        return SPTRSV_ERR_INVALID_ARG;
    }
}
