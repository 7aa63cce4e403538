/*
 * sptrsv_oracle.c — CPU restatement of the HCL-Fing/SPTRSV CSR SpTRSV path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the GPU library is
 * checked against.  Only the tests, the smoke check and the CPU-baseline leg
 * of the benchmark load it, and only as the checker or the timed CPU
 * baseline; the library never calls it.
 *
 * Every function restates the reference's algorithm and cites the reference
 * file:line it follows.  Pinned by: the reference's own known-answer test
 * (unit-valued L, b = row sums, x == 1 exactly; main.cu:228,236,
 * test.cu:10-15, header/matrix_properties.h:14) and by golden analysis and
 * solve vectors produced by the reference's own kernels built from source.
 *
 * Matrix convention: square lower-triangular CSR, 0-based, columns strictly
 * increasing, diagonal last in each row (main.cu:224-240).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Analysis                                                                  */
/* ------------------------------------------------------------------------ */

/* Level of every row, 1-based: level[i] = 1 + max(level[j]) over the
 * off-diagonal columns j of row i, 1 for rows with none.  Restates the
 * sync-free level kernel analysis/analysis_csr.cu:104-185 (the max
 * reduction at :172-175, the write 1 + my_level at :181).  Natural row order
 * is a topological order of a lower-triangular matrix, so one serial pass
 * suffices.  Returns nlevs = max level (analysis_csr.cu:305), 0 for n == 0. */
int oracle_levels(int n, const int* rowptr, const int* colidx, int* level)
{
    int nlevs = 0;
    for (int i = 0; i < n; i++) {
        int m = 0;
        for (int p = rowptr[i]; p < rowptr[i + 1] - 1; p++) {
            int l = level[colidx[p]];
            if (l > m) m = l;
        }
        level[i] = 1 + m;
        if (level[i] > nlevs) nlevs = level[i];
    }
    return nlevs;
}

/* Row bucket from the off-diagonal count (vect_size_calculator,
 * analysis_csr.cu:12-32; the count is rowptr[i+1]-rowptr[i]-1, :311-316). */
int oracle_bucket(int nnz_offdiag)
{
    if (nnz_offdiag == 0) return 6;
    if (nnz_offdiag == 1) return 0;
    if (nnz_offdiag <= 2) return 1;
    if (nnz_offdiag <= 4) return 2;
    if (nnz_offdiag <= 8) return 3;
    if (nnz_offdiag <= 16) return 4;
    return 5;
}

/* Lanes per row of a bucket (get_size_from_pos, analysis_csr.cu:84-102):
 * 1,2,4,8,16,32 for buckets 0..5 and -1 for the diagonal-only bucket 6. */
int oracle_lanes_of_bucket(int b)
{
    return b == 6 ? -1 : (1 << b);
}

/* iorder and the per-key counts.  key = 7*(level-1) + bucket
 * (get_index_from_size, analysis_csr.cu:53-57, applied at :322-332);
 * buckets[k] = number of rows with key k for k < 7*nlevs, buckets[7*nlevs] = 0
 * (stable_sort + reduce_by_key + scatter, :336-348); iorder = rows stably
 * sorted by key, ties in ascending row order (stable_sort_by_key of the keys
 * with 0..n-1, :350-352).  A counting sort that walks rows in ascending order
 * is stable by construction.  buckets must hold 7*nlevs+1 ints. */
void oracle_order(int n, const int* rowptr, const int* level, int nlevs, int* iorder, int* buckets)
{
    int nkeys = 7 * nlevs;
    memset(buckets, 0, sizeof(int) * (size_t)(nkeys + 1));
    int* key = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        int b = oracle_bucket(rowptr[i + 1] - rowptr[i] - 1);
        key[i] = 7 * (level[i] - 1) + b;
        buckets[key[i]]++;
    }
    int* cursor = (int*)malloc(sizeof(int) * (size_t)(nkeys + 1));
    int s = 0;
    for (int k = 0; k < nkeys; k++) {
        cursor[k] = s;
        s += buckets[k];
    }
    for (int i = 0; i < n; i++) iorder[cursor[key[i]]++] = i;
    free(cursor);
    free(key);
}

/* Number of multirow warps: sum over keys of ceil(count * lanes / 32) with
 * lanes -1 read as 1 (get_warps_per_bucks, analysis_csr.cu:66-71, summed by
 * the exclusive scan at :370-372). */
int oracle_n_warps(int nlevs, const int* buckets)
{
    long long w = 0;
    for (int k = 0; k < 7 * nlevs; k++) {
        int sz = oracle_lanes_of_bucket(k % 7);
        if (sz == -1) sz = 1;
        w += ((long long)buckets[k] * sz + 31) / 32;
    }
    return (int)w;
}

/* Multirow warp map (kernel_base, analysis_csr.cu:244-270, with the scans at
 * :370-374): for the x-th warp of key k, ivect_size_warp = lanes (0 for the
 * diagonal-only bucket) and ibase_row = (rows before key k) + x*(32/lanes')
 * where lanes' is lanes with 0 read as 1; ibase_row[n_warps] = n (:249).
 * ibase_row needs n_warps+1 ints, ivect_size_warp n_warps.  warp_lev, if not
 * NULL, receives the 1-based level of each warp. */
void oracle_warp_map(int n, int nlevs, const int* buckets, int* ibase_row, int* ivect_size_warp, int* warp_lev)
{
    int w = 0, rows = 0;
    for (int k = 0; k < 7 * nlevs; k++) {
        int cnt = buckets[k];
        int b = k % 7;
        int size = (b == 6) ? 0 : (1 << b);
        int sz = size == 0 ? 1 : size;
        int nw = (int)(((long long)cnt * sz + 31) / 32);
        for (int x = 0; x < nw; x++) {
            ivect_size_warp[w] = size;
            ibase_row[w] = rows + x * (32 / sz);
            if (warp_lev) warp_lev[w] = k / 7 + 1;
            w++;
        }
        rows += cnt;
    }
    ibase_row[w] = n;
}

/* ------------------------------------------------------------------------ */
/* Solve                                                                      */
/* ------------------------------------------------------------------------ */

/* Serial forward substitution in FP64, nrhs right-hand sides stored
 * row-major (value (i,k) at i*nrhs+k).  Restates the per-row arithmetic of
 * the reference kernels: left_sum = b_i - sum_j L_ij x_j, then
 * x_i = left_sum * (1/L_ii) (solver/solve_csr_simple.cu:45,60-106;
 * solve_csr_order.cu:239-278; solve_csr_multirow.cu:66-112).  The sum runs
 * in column order; the reference's per-lane partial sums reorder it, so
 * parity is a relative forward-error bound, not bitwise. */
void oracle_solve_f64(int n, const int* rowptr, const int* colidx, const double* val,
                      const double* b, double* x, int nrhs)
{
    for (int i = 0; i < n; i++) {
        int last = rowptr[i + 1] - 1;
        double piv = 1.0 / val[last];
        for (int k = 0; k < nrhs; k++) {
            double s = b[(size_t)i * nrhs + k];
            for (int p = rowptr[i]; p < last; p++) s -= val[p] * x[(size_t)colidx[p] * nrhs + k];
            x[(size_t)i * nrhs + k] = s * piv;
        }
    }
}

/* The reference's FP32 build (VALUE_TYPE = float, Makefile:7) restated:
 * values, b and x in float, piv = 1.0f / L_ii rounded in float, left_sum
 * accumulated in float in column order (solve_csr_simple.cu:45,60-106 with
 * VALUE_TYPE float).  x is returned widened to double. */
void oracle_solve_f32(int n, const int* rowptr, const int* colidx, const double* val,
                      const double* b, double* x, int nrhs)
{
    float* xf = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1) * (size_t)nrhs);
    for (int i = 0; i < n; i++) {
        int last = rowptr[i + 1] - 1;
        float piv = 1.0f / (float)val[last];
        for (int k = 0; k < nrhs; k++) {
            float s = (float)b[(size_t)i * nrhs + k];
            for (int p = rowptr[i]; p < last; p++) s -= (float)val[p] * xf[(size_t)colidx[p] * nrhs + k];
            xf[(size_t)i * nrhs + k] = s * piv;
        }
    }
    for (size_t t = 0; t < (size_t)n * nrhs; t++) x[t] = (double)xf[t];
    free(xf);
}

/* The same substitution carried in long double, the cross-check of the FP64
 * oracle (x_i = (b_i - sum) / L_ii, exact division). */
void oracle_solve_ld(int n, const int* rowptr, const int* colidx, const double* val,
                     const double* b, double* x, int nrhs)
{
    long double* xl = (long double*)malloc(sizeof(long double) * (size_t)(n > 0 ? n : 1) * (size_t)nrhs);
    for (int i = 0; i < n; i++) {
        int last = rowptr[i + 1] - 1;
        for (int k = 0; k < nrhs; k++) {
            long double s = b[(size_t)i * nrhs + k];
            for (int p = rowptr[i]; p < last; p++) s -= (long double)val[p] * xl[(size_t)colidx[p] * nrhs + k];
            xl[(size_t)i * nrhs + k] = s / (long double)val[last];
        }
    }
    for (size_t t = 0; t < (size_t)n * nrhs; t++) x[t] = (double)xl[t];
    free(xl);
}

/* Level-scheduled FP64 solve on all host threads: rows of one level are
 * independent, levels run in sequence.  Same arithmetic as oracle_solve_f64.
 * iorder/lev_ptr come from oracle_order (lev_ptr[l] = first iorder position
 * of level l+1, lev_ptr[nlevs] = n).  Used as the multi-core CPU baseline. */
void oracle_solve_levels_omp(int n, const int* rowptr, const int* colidx, const double* val,
                             const int* iorder, const int* lev_ptr, int nlevs,
                             const double* b, double* x, int nrhs)
{
    (void)n;
#pragma omp parallel
    {
        for (int l = 0; l < nlevs; l++) {
#pragma omp for schedule(static)
            for (int q = lev_ptr[l]; q < lev_ptr[l + 1]; q++) {
                int i = iorder[q];
                int last = rowptr[i + 1] - 1;
                double piv = 1.0 / val[last];
                for (int k = 0; k < nrhs; k++) {
                    double s = b[(size_t)i * nrhs + k];
                    for (int p = rowptr[i]; p < last; p++) s -= val[p] * x[(size_t)colidx[p] * nrhs + k];
                    x[(size_t)i * nrhs + k] = s * piv;
                }
            }
        }
    }
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* y = L x (all stored entries, diagonal included), row-major nrhs. */
void oracle_spmv(int n, const int* rowptr, const int* colidx, const double* val,
                 const double* x, double* y, int nrhs)
{
    for (int i = 0; i < n; i++)
        for (int k = 0; k < nrhs; k++) {
            double s = 0.0;
            for (int p = rowptr[i]; p < rowptr[i + 1]; p++) s += val[p] * x[(size_t)colidx[p] * nrhs + k];
            y[(size_t)i * nrhs + k] = s;
        }
}

/* max_i |a_i - b_i| / max_i |b_i| (relative forward error in the inf-norm). */
double oracle_rel_err_inf(size_t m, const double* a, const double* b)
{
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < m; i++) {
        double d = fabs(a[i] - b[i]);
        if (d != d) return INFINITY;
        if (d > num) num = d;
        if (fabs(b[i]) > den) den = fabs(b[i]);
    }
    return den > 0.0 ? num / den : num;
}
