/*
 * ORACLE (test infrastructure only): C restatement of the reference's CPU
 * direct solver, CpuSolver::solve_real / solve_complex
 * (src/solver/cpu.rs:28-96 and :98-171).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker / timed CPU baseline.
 *
 * Algorithm, as in the reference: CSR -> dense augmented matrix [A | b];
 * forward elimination with partial pivoting on |a_ik| (first maximum wins);
 * "singular matrix" when the pivot magnitude is < 1e-15; row swap; the
 * multiplier column is set to 0 and the rest of the row updated including
 * the rhs column; back substitution.  FP64, single thread.
 *
 * skip_zero_factors: see the elimination loop.
 * Return codes: 0 ok, 1 singular matrix, 2 dimension mismatch, 3 out of memory.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int oracle_dense_solve_real(int64_t n, int64_t ncols, const int64_t *row_ptr,
                            const int64_t *col, const double *val, int64_t nb,
                            const double *b, double *x, int skip_zero_factors)
{
    if (ncols != n || nb != n) return 2;                 /* cpu.rs:30-38 */
    if (n == 0) return 0;                                /* cpu.rs:39-41 */
    const int64_t w = n + 1;
    double *aug = (double *)calloc((size_t)n * (size_t)w, sizeof(double));
    double **row = (double **)malloc((size_t)n * sizeof(double *));
    if (!aug || !row) { free(aug); free(row); return 3; }
    for (int64_t i = 0; i < n; ++i) {                    /* to_dense + augment */
        row[i] = aug + i * w;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) row[i][col[k]] = val[k];
        row[i][n] = b[i];
    }
    for (int64_t k = 0; k < n; ++k) {                    /* cpu.rs:53-83 */
        double max_val = fabs(row[k][k]);
        int64_t max_row = k;
        for (int64_t i = k + 1; i < n; ++i) {
            double v = fabs(row[i][k]);
            if (v > max_val) { max_val = v; max_row = i; }
        }
        if (max_val < 1e-15) { free(aug); free(row); return 1; }
        if (max_row != k) { double *t = row[k]; row[k] = row[max_row]; row[max_row] = t; }
        const double pivot = row[k][k];
        const double *rk = row[k];
        for (int64_t i = k + 1; i < n; ++i) {
            double *ri = row[i];
            const double factor = ri[k] / pivot;
            ri[k] = 0.0;
            /* x - 0*y == x for finite y, so skipping is result-identical on
               finite data; the timed CPU baseline passes 0 and runs every update
               as the reference does. */
            if (skip_zero_factors && factor == 0.0) continue;
            for (int64_t j = k + 1; j <= n; ++j) ri[j] -= factor * rk[j];
        }
    }
    for (int64_t i = n - 1; i >= 0; --i) {               /* cpu.rs:86-93 */
        double sum = row[i][n];
        for (int64_t j = i + 1; j < n; ++j) sum -= row[i][j] * x[j];
        x[i] = sum / row[i][i];
    }
    free(aug);
    free(row);
    return 0;
}

/* cpu.rs:98-171: same elimination over Complex64, pivot on the norm |z|. */
int oracle_dense_solve_complex(int64_t n, int64_t ncols, const int64_t *row_ptr,
                               const int64_t *col, const double *val_ri, int64_t nb,
                               const double *b_ri, double *x_ri, int skip_zero_factors)
{
    if (ncols != n || nb != n) return 2;
    if (n == 0) return 0;
    const int64_t w = n + 1;
    double complex *aug = (double complex *)calloc((size_t)n * (size_t)w, sizeof(double complex));
    double complex **row = (double complex **)malloc((size_t)n * sizeof(double complex *));
    double complex *x = (double complex *)calloc((size_t)n, sizeof(double complex));
    if (!aug || !row || !x) { free(aug); free(row); free(x); return 3; }
    for (int64_t i = 0; i < n; ++i) {
        row[i] = aug + i * w;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            row[i][col[k]] = val_ri[2 * k] + I * val_ri[2 * k + 1];
        row[i][n] = b_ri[2 * i] + I * b_ri[2 * i + 1];
    }
    for (int64_t k = 0; k < n; ++k) {
        double max_val = cabs(row[k][k]);
        int64_t max_row = k;
        for (int64_t i = k + 1; i < n; ++i) {
            double v = cabs(row[i][k]);
            if (v > max_val) { max_val = v; max_row = i; }
        }
        if (max_val < 1e-15) { free(aug); free(row); free(x); return 1; }
        if (max_row != k) { double complex *t = row[k]; row[k] = row[max_row]; row[max_row] = t; }
        const double complex pivot = row[k][k];
        for (int64_t i = k + 1; i < n; ++i) {
            const double complex factor = row[i][k] / pivot;
            row[i][k] = 0.0;
            if (skip_zero_factors && factor == 0.0) continue;
            for (int64_t j = k + 1; j <= n; ++j) row[i][j] -= factor * row[k][j];
        }
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double complex sum = row[i][n];
        for (int64_t j = i + 1; j < n; ++j) sum -= row[i][j] * x[j];
        x[i] = sum / row[i][i];
    }
    for (int64_t i = 0; i < n; ++i) { x_ri[2 * i] = creal(x[i]); x_ri[2 * i + 1] = cimag(x[i]); }
    free(aug);
    free(row);
    free(x);
    return 0;
}
