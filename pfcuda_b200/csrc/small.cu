// small.cu -- Pfaffians of batches of small matrices (order n <= 32).
//
// Replaces the reference's small path: pf_sm_calc (src/pfaffian_sm.cu:4-99),
// one 32-thread block per matrix launched once per matrix by the XLA handler
// (bindings/jax_bindings.cu:107-109).  Same algorithm -- right-looking
// Parlett-Reid elimination with 2x2 pivots, pivot = first maximum of |row k|
// over the columns right of k (pfaffian_sm.cu:29-46), Pf = product of pivots
// times (-1)^(interchanges) (pfaffian_sm.cu:48-55,93-98) -- in a different
// shape:
//   * one persistent launch covers the whole batch;
//   * a group of G = 8, 16 or 32 lanes owns one matrix (32/G matrices per
//     warp), lane l keeps logical column l of the matrix in registers (G
//     values), so the O(n^3) rank-2 updates are register FMAs;
//   * the matrix is read once from HBM with coalesced row loads (each lane
//     takes its column's element of every row);
//   * column interchanges are relabelings of the owning lanes (no data moves),
//     row interchanges are register selects inside each lane;
//   * the pivot argmax is a shuffle butterfly on (|value|, column) so ties go
//     to the first column, as the reference's shuffle tree does
//     (pfaffian_sm.cu:36-46);
//   * the two pivot rows are broadcast through shared memory.
// A zero pivot ends the elimination with Pf = 0 (exact test; the reference
// uses |pivot| < 10 eps, include/pfaffian_utils.cuh:22-29).
//
// Column-major input is read through the same coalesced row loads: the row-major
// view of a column-major skew matrix is its transpose -A, and every operation
// of the elimination commutes exactly with negation, so the computed Pf is
// multiplied by (-1)^(n/2) at the end.
#include "common.cuh"
#include "small.cuh"

namespace pfb {

constexpr int kSmallThreads = 256;
constexpr int kSmallWarps = kSmallThreads / 32;

template <typename T>
PFB_D typename RealOf<T>::type pivot_key(T x)
{
    auto m = mag(x);
    return (m != m) ? (typename RealOf<T>::type)INFINITY : m;   // NaN is picked (and propagates)
}

// The column of the first maximum over the warp of (key >= 0, column): the
// largest key, and among equal keys the smallest column.
PFB_D unsigned first_max_col(double key, unsigned col)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(key);
    const unsigned hi = (unsigned)(b >> 32), lo = (unsigned)b;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    return __reduce_min_sync(0xffffffffu, (hi == mhi && lo == mlo) ? col : ~0u);
}
PFB_D unsigned first_max_col(float key, unsigned col)
{
    const unsigned b = (unsigned)__float_as_int(key);
    const unsigned m = __reduce_max_sync(0xffffffffu, b);
    return __reduce_min_sync(0xffffffffu, b == m ? col : ~0u);
}

template <typename T> PFB_D T phase_of(T a);
template <> PFB_D float phase_of(float a) { return a < 0.f ? -1.f : 1.f; }
template <> PFB_D double phase_of(double a) { return a < 0.0 ? -1.0 : 1.0; }
template <> PFB_D c64 phase_of(c64 a) { float m = hypotf(a.re, a.im); return mk(a.re / m, a.im / m); }
template <> PFB_D c128 phase_of(c128 a) { double m = hypot(a.re, a.im); return mk(a.re / m, a.im / m); }

template <typename T> struct PhaseAcc { using type = T; };
template <> struct PhaseAcc<c64> { using type = c128; };
template <> struct PhaseAcc<float> { using type = double; };

// The two pivot rows' entries of one column, broadcast to the group together.
template <typename T>
struct alignas(2 * sizeof(T)) XYPair {
    T x, y;
};

// R[1] <-> R[q] for a q in [LO, HI) that is the same for the whole warp: a
// binary search of uniform branches down to one register swap.
template <int LO, int HI, typename T, int G>
PFB_D void swap_row_at(T (&R)[G], int q)
{
    if constexpr (HI - LO == 1) {
        const T t = R[1];
        R[1] = R[LO];
        R[LO] = t;
    } else {
        constexpr int MID = (LO + HI) / 2;
        if (q < MID) swap_row_at<LO, MID>(R, q);
        else swap_row_at<MID, HI>(R, q);
    }
}

// One group of G lanes per matrix.  OUT_SLOG selects (log|Pf|, sign) output
// instead of the plain product.
//
// The pivot-step loop is a rolled loop over k: each lane's registers hold a
// window of its column, window position p = row k+p at step k, and the Schur
// update of row k+2+p writes window position p, so the window advances by two
// rows per step without extra moves and every register index is static.  (A
// fully unrolled elimination overflows the instruction cache at G = 32.)
template <typename T, int G, bool OUT_SLOG>
__global__ void __launch_bounds__(kSmallThreads, (sizeof(T) * G <= 256) ? 2 : 1)
pf_small_kernel(const T *__restrict__ A, int64_t batch, int n, int flip,
                T *__restrict__ out_val, double *__restrict__ out_log, T *__restrict__ out_sign)
{
    using Real = typename RealOf<T>::type;
    using Ph = typename PhaseAcc<T>::type;
    constexpr int MPW = 32 / G;   // matrices per warp

    __shared__ XYPair<T> s_xy[kSmallWarps][32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int gl = lane % G;            // lane within the group = initial column
    const int grp = lane / G;
    XYPair<T> *XY = &s_xy[warp][grp * G];
    const unsigned gmask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);

    const int64_t nn = (int64_t)n * n;
    const int64_t total_warps = (int64_t)gridDim.x * kSmallWarps;

    for (int64_t w = (int64_t)blockIdx.x * kSmallWarps + warp; w * MPW < batch; w += total_warps) {
        const int64_t m = w * MPW + grp;
        const bool valid = m < batch;
        const T *Am = A + (valid ? m : 0) * nn;

        T R[G];
#pragma unroll
        for (int r = 0; r < G; r++)
            R[r] = (valid && r < n && gl < n) ? ldg(&Am[(int64_t)r * n + gl]) : zero<T>();

        int lbl = gl;          // logical column held by this lane
        bool dead = !valid;    // zero pivot met (or no matrix)
        int swaps = 0;
        T prod = one<T>();
        double la = 0.0;
        Ph ph = one<Ph>();

#pragma unroll 1
        for (int k = 0; k < n - 1; k += 2) {
            // ---- pivot: first maximum of |A[k][c]| over logical columns c > k
            const bool cand = lbl > k && lbl < n;
            Real key = cand ? pivot_key(R[0]) : (Real)(-1);
            int col = lbl;
            if constexpr (G == 32) {
                // one matrix per warp: warp reductions (redux.sync) on the key's
                // bits -- a non-negative float compares as its bits -- then the
                // smallest column among the equal keys; a lane without a
                // candidate offers key 0 and column ~0, so it loses every tie
                col = (int)first_max_col(cand ? key : (Real)0, cand ? (unsigned)lbl : ~0u);
            } else {
#pragma unroll
                for (int off = G / 2; off > 0; off >>= 1) {
                    Real k2 = shfl_xor(key, off, G);
                    int c2 = shfl_xor(col, off, G);
                    if (k2 > key || (k2 == key && c2 < col)) { key = k2; col = c2; }
                }
            }
            const int j = col;
            const unsigned ball = __ballot_sync(0xffffffffu, lbl == j);
            const int src = __ffs((ball >> (grp * G)) & gmask) - 1;
            const T a = shfl(R[0], src, G);
            dead = dead || is_zero(a);

            // ---- interchange k+1 <-> j: columns by relabel; rows inside the
            // update below (window position q = j - k takes the old row k+1,
            // row k+1 becomes the old row j)
            const int q = j - k;
            T r1 = R[1], rq = r1;
            if constexpr (G == 32) {
                // one matrix per warp: q is warp-uniform, the rows swap in place
                if (q >= 2 && q < G) swap_row_at<2, G>(R, q);
                rq = R[1];
            } else {
#pragma unroll
                for (int p = 2; p < G; p++) rq = (p == q) ? R[p] : rq;
            }
            if (!dead && j != k + 1) {
                lbl = (lbl == k + 1) ? j : ((lbl == j) ? k + 1 : lbl);
                swaps ^= 1;
            }
            if (!dead) {
                if (OUT_SLOG) {
                    la += log((double)mag(a));
                    ph = ph * conv<Ph>(phase_of(a));
                } else {
                    prod = prod * a;
                }
            }

            // ---- rank-2 Schur update S[r][c] -= (x_r y_c - y_r x_c) / a, row
            // k+2+p into window position p
            XY[lbl] = XYPair<T>{R[0], rq};
            __syncwarp();
            if (!dead && lbl > k + 1 && lbl < n) {
                const T ia = recip(a);
                const T xh = R[0] * ia;
                const T yh = rq * ia;
                // chunks of 4 rows: the compiler barrier keeps it from hoisting
                // every shared-memory load of the step (register pressure);
                // chunks wholly below row n - 1 are skipped by a branch that is
                // uniform across the group (k, n are), so the step issues only
                // the rows it updates -- half of the fixed window on average
#pragma unroll
                for (int p0 = 0; p0 < G - 2; p0 += 4) {
                    if (k + 2 + p0 >= n) break;
#pragma unroll
                    for (int p = p0; p < p0 + 4 && p < G - 2; p++) {
                        const int r = k + 2 + p;
                        // (G = 32 swapped already; otherwise position q takes the old row k+1)
                        const T old = (G < 32 && p + 2 == q) ? r1 : R[p + 2];
                        if (r < n) {
                            const XYPair<T> v = XY[r];
                            R[p] = fma_(v.y, xh, fms_(v.x, yh, old));
                        }
                    }
                    asm volatile("" ::: "memory");
                }
            }
            __syncwarp();
        }

        if (valid && gl == 0) {
            const bool neg = (swaps ^ (flip & (n >> 1))) & 1;
            if (OUT_SLOG) {
                if (dead || n == 0 || (n & 1)) {
                    out_log[m] = -INFINITY;
                    out_sign[m] = zero<T>();
                } else {
                    out_log[m] = la;
                    Ph s = neg ? -ph : ph;
                    out_sign[m] = conv<T>(s);
                }
            } else {
                if (dead || n == 0 || (n & 1)) out_val[m] = zero<T>();
                else out_val[m] = neg ? -prod : prod;
            }
        }
    }
}

template <typename T, bool SLOG>
static int launch_small_t(const void *A, int64_t batch, int n, int layout, void *out_val,
                          double *out_log, void *out_sign, cudaStream_t stream)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int G = n <= 8 ? 8 : (n <= 16 ? 16 : 32);
    const int64_t mpw = 32 / G;
    const int64_t warps = (batch + mpw - 1) / mpw;
    int64_t blocks = (warps + kSmallWarps - 1) / kSmallWarps;
    const int64_t cap = (int64_t)sms * 16;   // grid-stride beyond 16 blocks per SM
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    const int flip = layout == PFB_COL_MAJOR ? 1 : 0;
    const T *a = static_cast<const T *>(A);
    T *ov = static_cast<T *>(out_val);
    T *os = static_cast<T *>(out_sign);
    dim3 grid((unsigned)blocks), block(kSmallThreads);
    if (G == 8)
        pf_small_kernel<T, 8, SLOG><<<grid, block, 0, stream>>>(a, batch, n, flip, ov, out_log, os);
    else if (G == 16)
        pf_small_kernel<T, 16, SLOG><<<grid, block, 0, stream>>>(a, batch, n, flip, ov, out_log, os);
    else
        pf_small_kernel<T, 32, SLOG><<<grid, block, 0, stream>>>(a, batch, n, flip, ov, out_log, os);
    return launch_status();
}

int launch_small(int dtype, bool slog, const void *A, int64_t batch, int n, int layout,
                 void *out_val, double *out_log, void *out_sign, cudaStream_t stream)
{
    switch (dtype) {
    case PFB_F32:
        return slog ? launch_small_t<float, true>(A, batch, n, layout, out_val, out_log, out_sign, stream)
                    : launch_small_t<float, false>(A, batch, n, layout, out_val, out_log, out_sign, stream);
    case PFB_F64:
        return slog ? launch_small_t<double, true>(A, batch, n, layout, out_val, out_log, out_sign, stream)
                    : launch_small_t<double, false>(A, batch, n, layout, out_val, out_log, out_sign, stream);
    case PFB_C64:
        return slog ? launch_small_t<c64, true>(A, batch, n, layout, out_val, out_log, out_sign, stream)
                    : launch_small_t<c64, false>(A, batch, n, layout, out_val, out_log, out_sign, stream);
    case PFB_C128:
        return slog ? launch_small_t<c128, true>(A, batch, n, layout, out_val, out_log, out_sign, stream)
                    : launch_small_t<c128, false>(A, batch, n, layout, out_val, out_log, out_sign, stream);
    default:
        return PFB_ERR_INVALID;
    }
}

}  // namespace pfb
