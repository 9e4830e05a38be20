// split.cuh -- the split-precision trailing update (error-free int8 slices on
// the tcgen05 tensor cores), see split.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "common.cuh"

namespace pfb {

struct MatState;

// Everything the panel kernel needs to write the slices of its Gauss vectors.
struct SplitArgs {
    int enabled;
    int n, k0, nb, kk;        // kk = K of the int8 products (nb real, 2*nb complex)
    int slices;               // number of 7-bit slices per operand
    int64_t mstride;          // elements per matrix in xs / ys (= slices * n * kk)
    int8_t *xs;               // [B][slices][n][kk]  A operand, K-major, rows = trailing index
    int8_t *ys;               // [B][slices][n][kk]  B operand
    int32_t *ex;              // [B][n] power-of-two exponent per trailing index
};

size_t split_workspace_bytes(bool cplx, int64_t batch, int n, int nb);
SplitArgs split_args(bool use, unsigned char *ws, bool cplx, int64_t batch, int n, int nb, int k0);
bool split_available();
int launch_split_update(bool cplx, void *W, int n, int k0, int K, int64_t batch,
                        const MatState *st, const SplitArgs &sa, cudaStream_t stream);

// Slice one trailing column's K panel values into `slices` int8 digits with a
// shared power-of-two scale (error-free: every digit and remainder is exact in
// FP64).  Y's digits are X's with each (u, w) pair mapped to (w, -u).  R is
// consumed (overwritten by the remainders).
template <typename T, int NB>
PFB_D void split_panel_column(const SplitArgs &sa, int64_t b, int col_rel, T (&R)[NB], int K)
{
    if (!sa.enabled) return;
    const int a = sa.k0 + sa.nb + col_rel;   // absolute trailing index
    double mx = 0.0;
#pragma unroll
    for (int r = 0; r < NB; r++) {
        if constexpr (IsComplex<T>::value) mx = fmax(mx, fmax(fabs(R[r].re), fabs(R[r].im)));
        else mx = fmax(mx, fabs(R[r]));
    }
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);          // mx < 2^e
    sa.ex[b * sa.n + a] = e;
    const double sc = ldexp(1.0, -e);
#pragma unroll
    for (int r = 0; r < NB; r++) {
        if (r >= K) R[r] = zero<T>();
        if constexpr (IsComplex<T>::value) { R[r].re *= sc; R[r].im *= sc; }
        else R[r] *= sc;
    }
    constexpr int KK = IsComplex<T>::value ? 2 * NB : NB;
    for (int s = 0; s < sa.slices; s++) {
        int8_t *xd = sa.xs + b * sa.mstride + ((int64_t)s * sa.n + a) * sa.kk;
        int8_t *yd = sa.ys + b * sa.mstride + ((int64_t)s * sa.n + a) * sa.kk;
#pragma unroll
        for (int r0 = 0; r0 < KK; r0 += 16) {
            alignas(16) int8_t dx[16], dy[16];
#pragma unroll
            for (int r = 0; r < 16; r++) {
                double v;
                if constexpr (IsComplex<T>::value) v = ((r0 + r) < NB ? R[r0 + r].re : R[r0 + r - NB].im);
                else v = R[r0 + r];
                v *= 128.0;
                const double d = trunc(v);
                if constexpr (IsComplex<T>::value) {
                    if ((r0 + r) < NB) R[r0 + r].re = v - d; else R[r0 + r - NB].im = v - d;
                } else {
                    R[r0 + r] = v - d;
                }
                dx[r] = (int8_t)d;
            }
            // X = [Re | Im] per column; Y pairs (u, w) -> (w, -u)
#pragma unroll
            for (int r = 0; r < 16; r += 2) {
                dy[r] = dx[r + 1];
                dy[r + 1] = (int8_t)(-dx[r]);
            }
            *reinterpret_cast<int4 *>(xd + r0) = *reinterpret_cast<const int4 *>(dx);
            *reinterpret_cast<int4 *>(yd + r0) = *reinterpret_cast<const int4 *>(dy);
        }
    }
}

}  // namespace pfb
