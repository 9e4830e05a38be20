// dmma.cuh -- FP64 tensor-core (DMMA) pieces of the skew rank-K trailing
// updates
//     S[a][b] += sum_r X[r][a] * Y[r][b],   Y[2s] = X[2s+1], Y[2s+1] = -X[2s],
// X = the K panel rows (real FP64).  One warp-wide mma.sync m8n8k4 does 256
// fused multiply-adds from two operand registers per lane, so the operand
// traffic from shared memory is a small fraction of the FFMA form's and the
// FP64 pipe, not the shared-memory port, bounds the update.
#pragma once
#include "common.cuh"

namespace pfb {

// D = A (8 x 4) * B (4 x 8) + D in FP64.  Lane l = 4g + t holds
// a = A[g][t], b = B[t][g] and d = D[g][2t .. 2t+1].
PFB_D void dmma_884(double (&d)[2], double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// 16-byte asynchronous global -> shared copy; the destination is zero-filled
// when !ok (src is then not read).
PFB_D void cp_async16(void *dst_smem, const void *src, bool ok)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(ok ? 16 : 0)
                 : "memory");
}
PFB_D void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> PFB_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Upper-triangle block (I, J), J >= I, of an nb x nb block grid from its
// linear index (row-major over the upper triangle).
PFB_D void upper_block(int idx, int nb, int &I, int &J)
{
    int i = 0;
    while (idx >= nb - i) {
        idx -= nb - i;
        i++;
    }
    I = i;
    J = i + idx;
}

// C fragments of an (8*MI) x (8*NJ) block with top-left (a0, b0) of the
// row-major n x n matrix W: lane (g, t) of fragment (i, j) holds
// W[a0 + 8i + g][b0 + 8j + 2t .. +1]; zero outside the matrix.  (n and b0
// even, so the pair is 16-byte aligned and lies wholly inside or outside.)
template <int MI, int NJ>
PFB_D void load_c_frags(double (&c)[MI][NJ][2], const double *__restrict__ W, int n, int a0, int b0)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
#pragma unroll
    for (int i = 0; i < MI; i++) {
        const int ar = a0 + 8 * i + g;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int bc = b0 + 8 * j + 2 * t;
            if (ar < n && bc < n) {
                const double2 v = *reinterpret_cast<const double2 *>(W + (int64_t)ar * n + bc);
                c[i][j][0] = v.x;
                c[i][j][1] = v.y;
            } else {
                c[i][j][0] = 0.0;
                c[i][j][1] = 0.0;
            }
        }
    }
}

// Store of the fragments back, strictly above the diagonal only (the lower
// triangle of the working matrix is never read).
template <int MI, int NJ>
PFB_D void store_c_frags(const double (&c)[MI][NJ][2], double *__restrict__ W, int n, int a0, int b0)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
#pragma unroll
    for (int i = 0; i < MI; i++) {
        const int ar = a0 + 8 * i + g;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int bc = b0 + 8 * j + 2 * t;
            if (ar < n && bc < n) {
                double *p = W + (int64_t)ar * n + bc;
                if (bc > ar) *reinterpret_cast<double2 *>(p) = make_double2(c[i][j][0], c[i][j][1]);
                else if (bc == ar) p[1] = c[i][j][1];
            }
        }
    }
}

// One k-step of 4 panel rows (kb, a multiple of 4): c += X^T Y over the
// (8*MI) x (8*NJ) block.  xs points at X[kb][a-offset], ys at the rows that
// Y is made of, X[kb][b-offset]; ld is the row stride of both, in doubles.
// Lane (g, t) reads X[kb+t][8i+g] and Y[kb+t][8j+g] = +-X[(kb+t)^1][8j+g]
// (negative for odd rows, i.e. odd t).  An 8-byte shared load is served per
// half-warp (g < 4, then g >= 4: four rows of four doubles each); a row stride
// of 4 (mod 16) doubles puts the four rows on distinct banks, so each fragment
// read is two conflict-free wavefronts.
template <int MI, int NJ>
PFB_D void dmma_kstep(double (&c)[MI][NJ][2], const double *xs, const double *ys, int ld)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    const double *xr = xs + t * ld + g;
    const double *yr = ys + (t ^ 1) * ld + g;
    double af[MI], bf[NJ];
#pragma unroll
    for (int i = 0; i < MI; i++) af[i] = xr[8 * i];
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        const double v = yr[8 * j];
        bf[j] = (t & 1) ? -v : v;
    }
#pragma unroll
    for (int i = 0; i < MI; i++)
#pragma unroll
        for (int j = 0; j < NJ; j++) dmma_884(c[i][j], af[i], bf[j]);
}

// ---- complex128: four real products per complex product,
//      re += ar br - ai bi,  im += ar bi + ai br.

// C fragments of an (8*MI) x (8*NJ) complex block: lane (g, t) of fragment
// (i, j) holds the real and imaginary parts of W[a0 + 8i + g][b0 + 8j + 2t .. +1]
// (two 16-byte elements); zero outside the matrix.
template <int MI, int NJ>
PFB_D void load_c_frags(double (&cr)[MI][NJ][2], double (&ci)[MI][NJ][2], const c128 *__restrict__ W, int n,
                        int a0, int b0)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
#pragma unroll
    for (int i = 0; i < MI; i++) {
        const int ar = a0 + 8 * i + g;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int bc = b0 + 8 * j + 2 * t;
            if (ar < n && bc < n) {
                const double2 *p = reinterpret_cast<const double2 *>(W + (int64_t)ar * n + bc);
                const double2 v0 = p[0], v1 = p[1];
                cr[i][j][0] = v0.x;
                ci[i][j][0] = v0.y;
                cr[i][j][1] = v1.x;
                ci[i][j][1] = v1.y;
            } else {
                cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
            }
        }
    }
}

template <int MI, int NJ>
PFB_D void store_c_frags(const double (&cr)[MI][NJ][2], const double (&ci)[MI][NJ][2], c128 *__restrict__ W,
                         int n, int a0, int b0)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
#pragma unroll
    for (int i = 0; i < MI; i++) {
        const int ar = a0 + 8 * i + g;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int bc = b0 + 8 * j + 2 * t;
            if (ar < n && bc < n) {
                double2 *p = reinterpret_cast<double2 *>(W + (int64_t)ar * n + bc);
                if (bc > ar) p[0] = make_double2(cr[i][j][0], ci[i][j][0]);
                if (bc + 1 > ar) p[1] = make_double2(cr[i][j][1], ci[i][j][1]);
            }
        }
    }
}

// One complex k-step of 4 rows (kb a multiple of 4): c += X^T Y over the
// block, X and Y as for dmma_kstep (with PAIRSWAP, Y[r] = +-X[r^1]; without,
// ys points at Y's own rows).  A 16-byte shared load is served per quarter
// warp (two columns of four rows); a row stride of 2 (mod 8) complex elements
// puts the eight on distinct bank groups.
template <int MI, int NJ, bool PAIRSWAP>
PFB_D void zdmma_kstep(double (&cr)[MI][NJ][2], double (&ci)[MI][NJ][2], const c128 *xs, const c128 *ys, int ld)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    const c128 *xr = xs + t * ld + g;
    const c128 *yr = ys + (PAIRSWAP ? (t ^ 1) : t) * ld + g;
    double ar[MI], ai[MI], nai[MI], br[NJ], bi[NJ];
#pragma unroll
    for (int i = 0; i < MI; i++) {
        const c128 v = xr[8 * i];
        ar[i] = v.re;
        ai[i] = v.im;
        nai[i] = -v.im;
    }
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        const c128 v = yr[8 * j];
        const bool neg = PAIRSWAP && (t & 1);
        br[j] = neg ? -v.re : v.re;
        bi[j] = neg ? -v.im : v.im;
    }
#pragma unroll
    for (int i = 0; i < MI; i++)
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            dmma_884(cr[i][j], ar[i], br[j]);
            dmma_884(cr[i][j], nai[i], bi[j]);
            dmma_884(ci[i][j], ar[i], bi[j]);
            dmma_884(ci[i][j], ai[i], br[j]);
        }
}

// ---- general products c += A B (the adjoint's kernels): A and B in shared
// memory, each either k-major (AK / BK: A[k][a], B[k][b]) or k-contiguous
// (A[a][k], B[b][k]).  Conflict-free row strides: real, 4 (mod 16) doubles in
// both layouts; complex, 2 (mod 8) elements k-major and 4 (mod 8)
// k-contiguous (16-byte loads are served per quarter warp).

template <int MI, int NJ, bool AK, bool BK>
PFB_D void dmma_kstep_g(double (&c)[MI][NJ][2], const double *A, int lda, const double *B, int ldb, int kb)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    double af[MI], bf[NJ];
#pragma unroll
    for (int i = 0; i < MI; i++) af[i] = AK ? A[(kb + t) * lda + 8 * i + g] : A[(8 * i + g) * lda + kb + t];
#pragma unroll
    for (int j = 0; j < NJ; j++) bf[j] = BK ? B[(kb + t) * ldb + 8 * j + g] : B[(8 * j + g) * ldb + kb + t];
#pragma unroll
    for (int i = 0; i < MI; i++)
#pragma unroll
        for (int j = 0; j < NJ; j++) dmma_884(c[i][j], af[i], bf[j]);
}

template <int MI, int NJ, bool AK, bool BK>
PFB_D void zdmma_kstep_g(double (&cr)[MI][NJ][2], double (&ci)[MI][NJ][2], const c128 *A, int lda,
                         const c128 *B, int ldb, int kb)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    double ar[MI], ai[MI], nai[MI], br[NJ], bi[NJ];
#pragma unroll
    for (int i = 0; i < MI; i++) {
        const c128 v = AK ? A[(kb + t) * lda + 8 * i + g] : A[(8 * i + g) * lda + kb + t];
        ar[i] = v.re;
        ai[i] = v.im;
        nai[i] = -v.im;
    }
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        const c128 v = BK ? B[(kb + t) * ldb + 8 * j + g] : B[(8 * j + g) * ldb + kb + t];
        br[j] = v.re;
        bi[j] = v.im;
    }
#pragma unroll
    for (int i = 0; i < MI; i++)
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            dmma_884(cr[i][j], ar[i], br[j]);
            dmma_884(cr[i][j], nai[i], bi[j]);
            dmma_884(ci[i][j], ar[i], bi[j]);
            dmma_884(ci[i][j], ai[i], br[j]);
        }
}

// Accumulators of an (8*MI) x (8*NJ) block for T = double or c128, with the
// k-step and element access the adjoint's kernels use; lane (g, t) of
// fragment (i, j) holds elements (8i + g, 8j + 2t + e), e = 0, 1.
template <typename T, int MI, int NJ> struct FragAcc;
template <int MI, int NJ> struct FragAcc<double, MI, NJ> {
    double c[MI][NJ][2];
    PFB_D void zero()
    {
#pragma unroll
        for (int i = 0; i < MI; i++)
#pragma unroll
            for (int j = 0; j < NJ; j++) c[i][j][0] = c[i][j][1] = 0.0;
    }
    template <bool AK, bool BK>
    PFB_D void step(const double *A, int lda, const double *B, int ldb, int kb)
    {
        dmma_kstep_g<MI, NJ, AK, BK>(c, A, lda, B, ldb, kb);
    }
    PFB_D double get(int i, int j, int e) const { return c[i][j][e]; }
};
template <int MI, int NJ> struct FragAcc<c128, MI, NJ> {
    double cr[MI][NJ][2], ci[MI][NJ][2];
    PFB_D void zero()
    {
#pragma unroll
        for (int i = 0; i < MI; i++)
#pragma unroll
            for (int j = 0; j < NJ; j++) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
    }
    template <bool AK, bool BK>
    PFB_D void step(const c128 *A, int lda, const c128 *B, int ldb, int kb)
    {
        zdmma_kstep_g<MI, NJ, AK, BK>(cr, ci, A, lda, B, ldb, kb);
    }
    PFB_D c128 get(int i, int j, int e) const { return mk(cr[i][j][e], ci[i][j][e]); }
};

}  // namespace pfb
