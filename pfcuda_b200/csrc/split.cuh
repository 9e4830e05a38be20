// split.cuh -- the split-precision trailing update (error-free int8 slices on
// the tcgen05 tensor cores), see split.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "common.cuh"

namespace pfb {

struct MatState;

constexpr int kSplitMaxSlices = 7;
constexpr int kSplitTileM = 128;   // rows of an operand chunk (the MMA M)

// Everything the panel kernel needs to write the int8 operands of the update.
//
// Operand layout: for slice s and 128-row tile t of the trailing index, one
// contiguous chunk of 128 * kk bytes in the tcgen05 "K-major, no swizzle"
// canonical form: core matrices of 8 rows x 16 bytes (128 contiguous bytes),
// the core matrix of row group g and K-group kc at byte (g * kk/16 + kc) * 128.
// A chunk is therefore the exact shared-memory image of an MMA operand tile and
// moves with one bulk copy.
struct SplitArgs {
    int enabled;
    int n, k0, nb, kk;        // kk = K of the int8 products (nb real, 2*nb complex)
    int slices;               // digits per operand (<= kSplitMaxSlices)
    int ntile;                // 128-row tiles covering the trailing index range
    int cplx;
    int64_t mstride;          // bytes per matrix of one operand array
    int8_t *xs;               // A operand: [B][slices][ntile][128 * kk]
    int8_t *ys;               // B operand (real: Y; complex: [Yr | -Yi])
    int8_t *ys2;              // complex only: [Yi | Yr]
    int32_t *ex;              // [B][n] power-of-two exponent per trailing index
    int32_t *err;             // [B] device-side timeout flags of the update kernel
    int epilogue;             // PFB_EPILOGUE_ROUNDTRIP or PFB_EPILOGUE_REDUCE
    int fail_b;               // matrix (of this range) whose waits give up at once, -1: none
                              // (PFB_SPLIT_TEST_TIMEOUT, which exercises the timeout path)
};

size_t split_workspace_bytes(bool cplx, int64_t batch, int n, int nb);
SplitArgs split_args(bool use, unsigned char *ws, bool cplx, int64_t batch, int n, int nb, int k0,
                     int slices);
// The same arrays seen from matrix b0 on (a range of the batch).
inline SplitArgs split_shift(SplitArgs a, int64_t b0)
{
    a.xs += b0 * a.mstride;
    a.ys += b0 * a.mstride;
    if (a.ys2) a.ys2 += b0 * a.mstride;
    a.ex += b0 * (int64_t)a.n;
    a.err += b0;
    a.fail_b = (a.fail_b >= 0 && a.fail_b >= b0) ? (int)(a.fail_b - b0) : -1;
    return a;
}
bool split_available();
int launch_split_update(bool cplx, void *W, int n, int k0, int K, int64_t batch,
                        MatState *st, const SplitArgs &sa, cudaStream_t stream);

PFB_D void split_store16(int8_t *base, const SplitArgs &sa, int64_t b, int s, int ar, int kc,
                         const int8_t (&d)[16])
{
    const int tile = ar >> 7, i = ar & 127, g = i >> 3, r = i & 7;
    int8_t *p = base + b * sa.mstride +
                ((int64_t)s * sa.ntile + tile) * (int64_t)(kSplitTileM * sa.kk) +
                (g * (sa.kk >> 4) + kc) * 128 + r * 16;
    *reinterpret_cast<int4 *>(p) = *reinterpret_cast<const int4 *>(d);
}

// |d| < 2^51 truncated toward zero, as an integer, without the conversion
// pipe: the magic-number addition rounds to nearest (exactly), then one step
// back toward zero if that went past d.
PFB_D long long trunc_to_int(double d)
{
    const double big = 0x1.8p52;
    long long x = __double_as_longlong(d + big) - 0x4338000000000000LL;
    const double r = (d + big) - big;
    if (d >= 0.0) { if (r > d) x -= 1; }
    else { if (r < d) x += 1; }
    return x;
}

// Digit s (0 = most significant) of the 49-bit truncated magnitude, signed.
PFB_D int8_t digit_of(long long x, int s)
{
    const long long m = x < 0 ? -x : x;
    const int d = (int)((m >> (42 - 7 * s)) & 127);
    return (int8_t)(x < 0 ? -d : d);
}

// Ozaki's error-free splitting of one trailing column of the panel rows into
// `slices` int8 digits under a shared power-of-two scale: with e the exponent
// of the column's largest magnitude (column_exponent; mx < 2^e), every value x
// becomes X = trunc(x 2^(49-e)) (|X| < 2^49, exact: a power-of-two scaling and
// a truncation), and digit s is bits 42-7s .. 48-7s of |X| with x's sign --
// the same digits as repeated "multiply by 128, truncate, keep the remainder".
// Y's digits are X's with each (u, w) pair mapped to (w, -u).
template <typename T>
PFB_D double max_component(const T (&R)[16])
{
    double mx = 0.0;
#pragma unroll
    for (int r = 0; r < 16; r++) {
        if constexpr (IsComplex<T>::value) mx = fmax(mx, fmax(fabs(R[r].re), fabs(R[r].im)));
        else mx = fmax(mx, fabs(R[r]));
    }
    return mx;
}

PFB_D int column_exponent(double mx)
{
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    return e;
}

// Digits of rows 16 kc .. 16 kc + 15 of one column (R, scaled by sc = 2^(49-e))
// into the A image (and the B images) of the split update.
template <typename T, int NB>
PFB_D void split_chunk(const SplitArgs &sa, int64_t b, int col_rel, int kc, const T (&R)[16], double sc)
{
    if constexpr (!IsComplex<T>::value) {
        long long X[16];
#pragma unroll
        for (int r = 0; r < 16; r++) X[r] = trunc_to_int(R[r] * sc);
        for (int s = 0; s < sa.slices; s++) {
            alignas(16) int8_t dx[16];
            alignas(16) int8_t dy[16];
#pragma unroll
            for (int r = 0; r < 16; r++) dx[r] = digit_of(X[r], s);
#pragma unroll
            for (int r = 0; r < 16; r += 2) {   // (u, w) -> (w, -u)
                dy[r] = dx[r + 1];
                dy[r + 1] = (int8_t)(-dx[r]);
            }
            split_store16(sa.xs, sa, b, s, col_rel, kc, dx);
            split_store16(sa.ys, sa, b, s, col_rel, kc, dy);
        }
    } else {
        // A = [Xr | Xi],  B1 = [Yr | -Yi],  B2 = [Yi | Yr]:  Re = A.B1, Im = A.B2
        long long Xr[16], Xi[16];
#pragma unroll
        for (int r = 0; r < 16; r++) {
            Xr[r] = trunc_to_int(R[r].re * sc);
            Xi[r] = trunc_to_int(R[r].im * sc);
        }
        for (int s = 0; s < sa.slices; s++) {
            alignas(16) int8_t xr[16];
            alignas(16) int8_t xi[16];
            alignas(16) int8_t yr[16];
            alignas(16) int8_t yi[16];
            alignas(16) int8_t t[16];
#pragma unroll
            for (int r = 0; r < 16; r++) {
                xr[r] = digit_of(Xr[r], s);
                xi[r] = digit_of(Xi[r], s);
            }
#pragma unroll
            for (int r = 0; r < 16; r += 2) {
                yr[r] = xr[r + 1];
                yr[r + 1] = (int8_t)(-xr[r]);
                yi[r] = xi[r + 1];
                yi[r + 1] = (int8_t)(-xi[r]);
            }
            split_store16(sa.xs, sa, b, s, col_rel, kc, xr);
            split_store16(sa.xs, sa, b, s, col_rel, NB / 16 + kc, xi);
            split_store16(sa.ys, sa, b, s, col_rel, kc, yr);
#pragma unroll
            for (int r = 0; r < 16; r++) t[r] = (int8_t)(-yi[r]);
            split_store16(sa.ys, sa, b, s, col_rel, NB / 16 + kc, t);
            split_store16(sa.ys2, sa, b, s, col_rel, kc, yi);
            split_store16(sa.ys2, sa, b, s, col_rel, NB / 16 + kc, yr);
        }
    }
}

}  // namespace pfb
