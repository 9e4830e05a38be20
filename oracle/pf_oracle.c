/*
 * pf_oracle.c -- CPU oracle for the Pfaffian hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA engine is compared
 * against.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py load it; the engine itself never links, calls or falls back to it.
 *
 * It restates the reference's lazy (left-looking) Parlett-Reid recurrence with
 * 2x2 pivots:
 *   - real:    src/pfaffian_cpu.cpp:22-103 (row-major, strict upper triangle,
 *              lazy row update :32-45, first-max argmax :47-52, skew-aware
 *              swap :54-75, exact zero-pivot test :79-80, lazy update of row
 *              k+1 :85-98, scaling by the reciprocal pivot :100-102);
 *   - complex: the same recurrence, which pfcuda/pfaffian_py.py:17-50 runs for
 *              any dtype (there the scaled row is divided by the pivot, :48).
 * The one change is the accumulation: the reference multiplies pivots into a
 * plain product (pfaffian_cpu.cpp:63,74,83), which overflows or underflows for
 * large matrices.  Here log|pivot| is summed and the phase pivot/|pivot| is
 * multiplied in, so the result is (log|Pf|, sign).
 *
 * Pivot choice: the argmax runs over the UPDATED row k, as
 * pfcuda/pfaffian_py.py:29-32 and the reference's small CUDA kernel
 * (src/pfaffian_sm.cu:29-46) do.  src/pfaffian_cpu.cpp:29-30 instead reads
 * |A[k][k+1]| before the lazy update of row k and compares the updated
 * candidates against that stale value; pfo_pf_d_as_shipped keeps that and the
 * closed forms for n = 2, 4, and is bit-identical to the compiled reference.
 *
 * Build flags must include -ffp-contract=off so that no multiply-add is fused:
 * the reference is built without FMA (-O3, no -march), and the product mode
 * then matches it exactly.
 *
 * Every entry point works on a caller-owned row-major n x n array, which it
 * overwrites (as the reference does).  piv, when not NULL, receives the column
 * index chosen at each pivot step (n/2 entries).
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

#define RM(A, n, i, j) ((A)[(size_t)(i) * (size_t)(n) + (size_t)(j)])

/* ---------------------------------------------------------------- real f64 */

static int pf_core_d(double *A, int n, double *log_abs, double *sign,
                     double *prod, int32_t *piv, int stale)
{
    double la = 0.0, sg = 1.0, pr = 1.0;
    if (n == 0 || (n & 1)) {
        if (log_abs) *log_abs = -INFINITY;
        if (sign) *sign = 0.0;
        if (prod) *prod = 0.0;
        return 0;
    }
    for (int k = 0; k < n - 1; k += 2) {
        const int rows = k;
        double *v = &RM(A, n, k, 0);
        double *w = &RM(A, n, k + 1, 0);
        /* src/pfaffian_cpu.cpp:29-30 takes |A[k][k+1]| before the lazy update
           of row k; `stale` keeps that, otherwise the updated value is used */
        const double kv_stale = fabs(v[k + 1]);

        /* lazy update of row k (pfaffian_cpu.cpp:32-45) */
        for (int r = 0; r < rows; r += 2) {
            const double k0 = RM(A, n, r, k);
            const double k1 = -RM(A, n, r + 1, k);
            const double *r0 = &RM(A, n, r, 0);
            const double *r1 = &RM(A, n, r + 1, 0);
            for (int c = k + 1; c < n; c++) {
                const double c_r0 = r0[c];
                const double c_r1 = -r1[c];
                v[c] += (c_r1 * k0 - c_r0 * k1);
            }
        }

        /* first maximum of |row k| over columns > k (pfaffian_cpu.cpp:47-52,
           pfcuda/pfaffian_py.py:32) */
        int kp = k + 1;
        double kv = stale ? kv_stale : fabs(v[kp]);
        for (int c = k + 2; c < n; c++) {
            const double a = fabs(v[c]);
            if (a > kv) { kp = c; kv = a; }
        }
        if (piv) piv[k / 2] = kp;

        /* skew-aware interchange of k+1 and kp on the upper triangle
           (pfaffian_cpu.cpp:54-75) */
        if (kp != k + 1) {
            const int i = k + 1, j = kp;
            for (int r = 0; r < i; r++) {
                double t = RM(A, n, r, i); RM(A, n, r, i) = RM(A, n, r, j); RM(A, n, r, j) = t;
            }
            for (int c = j + 1; c < n; c++) {
                double t = RM(A, n, i, c); RM(A, n, i, c) = RM(A, n, j, c); RM(A, n, j, c) = t;
            }
            for (int m = i + 1; m < j; m++) {
                double t = RM(A, n, i, m);
                RM(A, n, i, m) = -RM(A, n, m, j);
                RM(A, n, m, j) = -t;
            }
            RM(A, n, i, j) = -RM(A, n, i, j);
            sg = -sg;
            pr *= -1.0;
        }

        const double pivot = v[k + 1];
        if (pivot == 0) {
            if (log_abs) *log_abs = -INFINITY;
            if (sign) *sign = 0.0;
            if (prod) *prod = 0.0;
            return 1;
        }
        const double f = 1.0 / pivot;
        pr *= pivot;
        la += log(fabs(pivot));
        if (pivot < 0) sg = -sg;

        /* lazy update of row k+1 (pfaffian_cpu.cpp:85-98) */
        for (int r = 0; r < rows; r += 2) {
            const double k0 = RM(A, n, r, k + 1);
            const double k1 = -RM(A, n, r + 1, k + 1);
            const double *r0 = &RM(A, n, r, 0);
            const double *r1 = &RM(A, n, r + 1, 0);
            for (int c = k + 2; c < n; c++) {
                const double c_r0 = r0[c];
                const double c_r1 = -r1[c];
                w[c] += (c_r1 * k0 - c_r0 * k1);
            }
        }
        /* scale row k into the Gauss vector (pfaffian_cpu.cpp:100-102) */
        for (int c = k + 2; c < n; c++) v[c] *= f;
    }
    if (log_abs) *log_abs = la;
    if (sign) *sign = sg;
    if (prod) *prod = pr;
    return 0;
}

/* log|Pf| and sign of one real matrix (overwrites A). */
int pfo_slog_d(double *A, int n, double *log_abs, double *sign, int32_t *piv)
{
    return pf_core_d(A, n, log_abs, sign, NULL, piv, 0);
}

/* Plain product of pivots, pivoting on the updated row (overwrites A). */
double pfo_pf_d(double *A, int n, int32_t *piv)
{
    double pr = 0.0;
    pf_core_d(A, n, NULL, NULL, &pr, piv, 0);
    return pr;
}

/*
 * Bit-for-bit restatement of src/pfaffian_cpu.cpp:7-106 as the reference
 * ships it: the closed forms for n = 2 and 4 (:11-20) and the stale first
 * candidate of the argmax (:29-30).  Used only to pin this file against the
 * compiled reference.
 */
double pfo_pf_d_as_shipped(double *A, int n)
{
    if (n == 0 || (n & 1)) return 0.0;
    if (n == 2) return RM(A, n, 0, 1);
    if (n == 4)
        return RM(A, n, 0, 1) * RM(A, n, 2, 3) - RM(A, n, 0, 2) * RM(A, n, 1, 3) +
               RM(A, n, 0, 3) * RM(A, n, 1, 2);
    double pr = 0.0;
    pf_core_d(A, n, NULL, NULL, &pr, NULL, 1);
    return pr;
}

/* ------------------------------------------------------------ complex c128 */

static int pf_core_z(double complex *A, int n, double *log_abs,
                     double complex *phase, double complex *prod, int32_t *piv)
{
    double la = 0.0;
    double complex ph = 1.0, pr = 1.0;
    if (n == 0 || (n & 1)) {
        if (log_abs) *log_abs = -INFINITY;
        if (phase) *phase = 0.0;
        if (prod) *prod = 0.0;
        return 0;
    }
    for (int k = 0; k < n - 1; k += 2) {
        double complex *v = &RM(A, n, k, 0);
        double complex *w = &RM(A, n, k + 1, 0);
        for (int r = 0; r < k; r += 2) {
            const double complex k0 = RM(A, n, r, k);
            const double complex k1 = -RM(A, n, r + 1, k);
            const double complex *r0 = &RM(A, n, r, 0);
            const double complex *r1 = &RM(A, n, r + 1, 0);
            for (int c = k + 1; c < n; c++)
                v[c] += ((-r1[c]) * k0 - r0[c] * k1);
        }
        /* np.abs(...).argmax() (pfaffian_py.py:32): first maximum of the modulus (hypot) */
        int kp = k + 1;
        double kv = cabs(v[kp]);
        for (int c = k + 2; c < n; c++) {
            const double a = cabs(v[c]);
            if (a > kv) { kp = c; kv = a; }
        }
        if (piv) piv[k / 2] = kp;
        if (kp != k + 1) {
            const int i = k + 1, j = kp;
            for (int r = 0; r < i; r++) {
                double complex t = RM(A, n, r, i); RM(A, n, r, i) = RM(A, n, r, j); RM(A, n, r, j) = t;
            }
            for (int c = j + 1; c < n; c++) {
                double complex t = RM(A, n, i, c); RM(A, n, i, c) = RM(A, n, j, c); RM(A, n, j, c) = t;
            }
            for (int m = i + 1; m < j; m++) {
                double complex t = RM(A, n, i, m);
                RM(A, n, i, m) = -RM(A, n, m, j);
                RM(A, n, m, j) = -t;
            }
            RM(A, n, i, j) = -RM(A, n, i, j);
            ph = -ph;
            pr = -pr;
        }
        const double complex pivot = v[k + 1];
        if (pivot == 0) {
            if (log_abs) *log_abs = -INFINITY;
            if (phase) *phase = 0.0;
            if (prod) *prod = 0.0;
            return 1;
        }
        const double ap = cabs(pivot);
        pr *= pivot;
        la += log(ap);
        ph *= pivot / ap;
        /* keep the phase on the unit circle over thousands of steps */
        if ((k & 63) == 62) ph /= cabs(ph);
        for (int r = 0; r < k; r += 2) {
            const double complex k0 = RM(A, n, r, k + 1);
            const double complex k1 = -RM(A, n, r + 1, k + 1);
            const double complex *r0 = &RM(A, n, r, 0);
            const double complex *r1 = &RM(A, n, r + 1, 0);
            for (int c = k + 2; c < n; c++)
                w[c] += ((-r1[c]) * k0 - r0[c] * k1);
        }
        /* pfaffian_py.py:48 divides the row by the pivot */
        for (int c = k + 2; c < n; c++) v[c] /= pivot;
    }
    if (log_abs) *log_abs = la;
    if (phase) *phase = ph / cabs(ph);
    if (prod) *prod = pr;
    return 0;
}

/* log|Pf| and unit phase of one complex matrix (interleaved re/im, overwrites A). */
int pfo_slog_z(double *A, int n, double *log_abs, double *phase_re_im, int32_t *piv)
{
    double complex ph = 0.0;
    int rc = pf_core_z((double complex *)A, n, log_abs, &ph, NULL, piv);
    if (phase_re_im) { phase_re_im[0] = creal(ph); phase_re_im[1] = cimag(ph); }
    return rc;
}

/* Plain complex product, the value pfcuda/pfaffian_py.py returns (overwrites A). */
void pfo_pf_z(double *A, int n, double *out_re_im, int32_t *piv)
{
    double complex pr = 0.0;
    pf_core_z((double complex *)A, n, NULL, NULL, &pr, piv);
    out_re_im[0] = creal(pr);
    out_re_im[1] = cimag(pr);
}

/* ------------------------------------------------------------------ batches */

/*
 * Batch drivers: B contiguous row-major n x n matrices, each copied to a
 * private scratch matrix first (the inputs are left untouched).  Matrices are
 * spread over OpenMP threads when the file is built with -fopenmp.
 */
int pfo_slog_batch_d(const double *A, int64_t B, int n, double *log_abs,
                     double *sign, int32_t *piv)
{
    const size_t nn = (size_t)n * (size_t)n;
    int bad = 0;
#pragma omp parallel
    {
        double *S = (double *)malloc(nn ? nn * sizeof(double) : 1);
        if (!S) {
#pragma omp atomic write
            bad = 1;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t b = 0; b < B; b++) {
                memcpy(S, A + (size_t)b * nn, nn * sizeof(double));
                pf_core_d(S, n, &log_abs[b], &sign[b], NULL,
                          piv ? piv + (size_t)b * (size_t)(n / 2) : NULL, 0);
            }
            free(S);
        }
    }
    return bad ? -1 : 0;
}

int pfo_slog_batch_z(const double *A, int64_t B, int n, double *log_abs,
                     double *phase_re_im, int32_t *piv)
{
    const size_t nn = (size_t)n * (size_t)n;
    int bad = 0;
#pragma omp parallel
    {
        double complex *S = (double complex *)malloc(nn ? nn * sizeof(double complex) : 1);
        if (!S) {
#pragma omp atomic write
            bad = 1;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t b = 0; b < B; b++) {
                double complex ph = 0.0;
                memcpy(S, A + 2 * (size_t)b * nn, nn * sizeof(double complex));
                pf_core_z(S, n, &log_abs[b], &ph, NULL,
                          piv ? piv + (size_t)b * (size_t)(n / 2) : NULL);
                phase_re_im[2 * b] = creal(ph);
                phase_re_im[2 * b + 1] = cimag(ph);
            }
            free(S);
        }
    }
    return bad ? -1 : 0;
}

int pfo_pf_batch_d(const double *A, int64_t B, int n, double *out, int as_shipped)
{
    const size_t nn = (size_t)n * (size_t)n;
    int bad = 0;
#pragma omp parallel
    {
        double *S = (double *)malloc(nn ? nn * sizeof(double) : 1);
        if (!S) {
#pragma omp atomic write
            bad = 1;
        } else {
#pragma omp for schedule(dynamic, 16)
            for (int64_t b = 0; b < B; b++) {
                double pr = 0.0;
                memcpy(S, A + (size_t)b * nn, nn * sizeof(double));
                if (as_shipped) pr = pfo_pf_d_as_shipped(S, n);
                else pf_core_d(S, n, NULL, NULL, &pr, NULL, 0);
                out[b] = pr;
            }
            free(S);
        }
    }
    return bad ? -1 : 0;
}

int pfo_num_threads(void)
{
    int t = 1;
#pragma omp parallel
    {
#pragma omp single
        {
#ifdef _OPENMP
            extern int omp_get_num_threads(void);
            t = omp_get_num_threads();
#endif
        }
    }
    return t;
}
