// large.cu -- (log|Pf|, sign) of large skew matrices by a blocked skew-LTL^T
// (Parlett-Reid) factorisation with 2x2 pivots.
//
// The reference's large path (src/slog_pfaffian_lg.cu:151-211) is the
// unblocked left-looking recurrence driven from the host: per pivot pair it
// launches row_update / argmax / swap_rows / swap_cols / apply_updates and
// copies the pivot back to the host (slog_pfaffian_lg.cu:178), so it is bound
// by ~2n launches and n/2 host round trips.  The mathematics kept from it:
//   * pivot step k (even): the updated row k, its first maximum in modulus over
//     the columns right of k picks j, rows/columns k+1 and j are interchanged,
//     the pivot is a = A[k][k+1] (slog_pfaffian_lg.cu:166-197);
//   * log|Pf| = sum log|a|, sign = prod a/|a| times (-1)^(interchanges)
//     (slog_pfaffian_lg.cu:186-194); a zero pivot gives (-inf, 0) (:180-184);
//   * the stored factors: row k keeps u = (updated row k)/a, row k+1 keeps
//     w = -(updated row k+1) (apply_updates, slog_pfaffian_lg.cu:136-149), so the
//     Schur complement is S = A22 + sum (u w^T - w u^T).
// The shape is new and runs entirely on the device:
//   * copy_in: the upper triangle of the input's row-major view (any dtype,
//     either layout) becomes an FP64 / complex128 working matrix W in the
//     workspace; nothing reads below its diagonal.
//   * panel_kernel (one thread-block cluster per matrix): NB pivot rows at a
//     time.  Each trailing column of the panel rows lives in the registers of
//     one thread, the NB x NB block of panel columns is replicated in every
//     CTA's shared memory, and a pivot step costs one cluster barrier: every CTA
//     pushes its best candidate (with that column's panel entries) into every
//     other CTA's shared memory before the barrier, so after it each CTA knows
//     the pivot and the interchanged column without another round trip.  Rows
//     are updated lazily within the panel (left-looking), exactly the
//     reference's recurrence restricted to the panel's own Gauss vectors.
//   * trailing update: S22 += X^T Y on the upper-triangle tiles, X = the NB panel
//     rows (u/w interleaved), Y = the same rows with each (u, w) pair replaced by
//     (w, -u) -- a skew rank-NB update, in FP64 on the FP64 tensor cores
//     (gemm_dmma_kernel; complex: gemm_zdmma_kernel) or in error-free int8
//     slices on the tcgen05 tensor cores (split.cu).
//   * finalize: log/sign from the per-matrix state.
// Column-major input is handled like the small path: its row-major view is the
// transpose -A, and Pf(-A) = (-1)^(n/2) Pf(A) exactly.
#include <limits.h>

#include <mutex>

#include "common.cuh"
#include "large.cuh"
#include "split.cuh"
#include "panel.cuh"
#include "dmma.cuh"
#include "tune_table.h"

namespace pfb {

// ---------------------------------------------------------- workspace layout

struct LargeLayout {
    size_t piv_off, st_off, w_off, split_off, total;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static bool large_cfg(int dtype, int n, int *nb, int *cpt)
{
    const bool cplx = dtype == PFB_C64 || dtype == PFB_C128;
    // trailing capacity of one panel launch: kClusterMax * kTT * cpt columns
    if (!cplx) {
        if (n <= kClusterMax * kTT + 64) { *nb = 64; *cpt = 1; return true; }
        if (n <= 2 * kClusterMax * kTT + 32) { *nb = 32; *cpt = 2; return true; }
    } else {
        if (n <= kClusterMax * kTT + 32) { *nb = 32; *cpt = 1; return true; }
    }
    return false;
}

static LargeLayout large_layout(int dtype, int64_t B, int n, int mode)
{
    LargeLayout L{};
    const bool cplx = dtype == PFB_C64 || dtype == PFB_C128;
    const size_t ts = cplx ? 16 : 8;
    int nb = 64, cpt = 1;
    large_cfg(dtype, n, &nb, &cpt);
    size_t off = 0;
    L.piv_off = off;
    off = align256(off + (size_t)B * (size_t)(n / 2) * sizeof(int32_t));
    L.st_off = off;
    off = align256(off + (size_t)B * sizeof(MatState));
    L.w_off = off;
    off = align256(off + (size_t)B * (size_t)n * (size_t)n * ts);
    L.split_off = off;
    if ((mode & 0xff) == PFB_MODE_SPLIT) off = align256(off + split_workspace_bytes(cplx, B, n, nb));
    L.total = off;
    return L;
}

int large_panel_width(int dtype, int n)
{
    int nb, cpt;
    return large_cfg(dtype, n, &nb, &cpt) ? nb : 0;
}

LargeView large_view(int dtype, int64_t batch, int n, int mode, void *workspace)
{
    const LargeLayout L = large_layout(dtype, batch, n, mode);
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    return LargeView{reinterpret_cast<int32_t *>(ws + L.piv_off), reinterpret_cast<MatState *>(ws + L.st_off),
                     ws + L.w_off};
}

size_t large_workspace_bytes(int dtype, int64_t batch, int n, int mode)
{
    int nb, cpt;
    if (n > 32 && !large_cfg(dtype, n, &nb, &cpt)) return 0;
    return large_layout(dtype, batch, n, mode).total;
}

// ----------------------------------------------------------------- copy in

// W <- A widened, the upper triangle only (diagonal included): nothing reads
// below the diagonal of W.  One warp per row at a time, the row's columns
// r .. n-1 in coalesced runs of 32.
// The matrices come either contiguous from A or, when Ap is set, one pointer
// per matrix (Ap[b], a device array).
template <typename S, typename T>
__global__ void copy_in_kernel(const S *__restrict__ A, const S *const *__restrict__ Ap, T *__restrict__ W,
                               int64_t batch, int n, MatState *st)
{
    const int lane = threadIdx.x & 31;
    const int64_t rows = batch * n;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t R = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; R < rows; R += nwarps) {
        const int r = (int)(R % n);
        const S *src = Ap ? Ap[R / n] + (int64_t)r * n : A + R * n;
        T *dst = W + R * n;
        for (int c = r + lane; c < n; c += 32) dst[c] = conv<T>(src[c]);
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < batch; b += stride) {
        MatState s;
        s.log_abs = 0.0;
        s.ph_re = 1.0;
        s.ph_im = 0.0;
        s.parity = 0;
        s.dead = 0;
        st[b] = s;
    }
}

template <typename T, int NB, int CPT>
__global__ void __launch_bounds__(kTT, 1)
panel_kernel(T *__restrict__ W_all, int n, int k0, MatState *__restrict__ st_all,
             int32_t *__restrict__ piv_all)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PanelSmem<T, NB> &sm = *reinterpret_cast<PanelSmem<T, NB> *>(smem_raw);
    const int64_t b = blockIdx.y;
    panel_body<T, NB, CPT>(sm, W_all + b * (int64_t)n * n, n, k0, st_all + b, piv_all + b * (int64_t)(n / 2));
}

// The same panel with half of each window in shared memory (panel_body_hs):
// at most 128 registers per thread, so two CTAs fit on an SM.
template <typename T, int NB>
__global__ void __launch_bounds__(kTT, 2)
panel_hs_kernel(T *__restrict__ W_all, int n, int k0, MatState *__restrict__ st_all,
                int32_t *__restrict__ piv_all)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PanelSmemHS<T, NB> &sm = *reinterpret_cast<PanelSmemHS<T, NB> *>(smem_raw);
    const int64_t b = blockIdx.y;
    panel_body_hs<T, NB>(sm, W_all + b * (int64_t)n * n, n, k0, st_all + b, piv_all + b * (int64_t)(n / 2));
}

// The int8 operand images of the split update for the panel at k0 (a full
// panel: its NB rows of W at the trailing columns hold the Gauss vectors).
// NB/16 adjacent threads share a trailing column, one 16-row chunk each: the
// column's exponent is the maximum over their chunks (lane shuffles), then
// each slices its chunk (split_chunk).  A launch of its own over every SM,
// rather than a tail of the panel kernel on the panel's CTAs only.
template <typename T, int NB>
__global__ void __launch_bounds__(256)
split_slice_kernel(const T *__restrict__ W_all, int n, int k0, const MatState *__restrict__ st_all, SplitArgs sa)
{
    constexpr int CH = NB / 16;        // threads per column
    constexpr int CPB = 256 / CH;      // columns per block
    static_assert(CH == 2 || CH == 4, "16-row chunks of a 32- or 64-row panel");
    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    const int k1 = k0 + NB;
    const int ch = threadIdx.x % CH;
    const int c = k1 + blockIdx.x * CPB + threadIdx.x / CH;
    const bool ok = c < n;
    const T *W = W_all + b * (int64_t)n * n;
    T R[16];
#pragma unroll
    for (int r = 0; r < 16; r++) R[r] = ok ? W[(int64_t)(k0 + 16 * ch + r) * n + c] : zero<T>();
    double mx = max_component(R);
#pragma unroll
    for (int off = 1; off < CH; off <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (!ok) return;
    const int e = column_exponent(mx);
    if (ch == 0) sa.ex[b * sa.n + c] = e;
    split_chunk<T, NB>(sa, b, c - k1, ch, R, ldexp(1.0, 49 - e));
}

// ------------------------------------------------------- FP64 trailing update

// S22[a][b] += sum_t X[t][a] * Y[t][b] over the upper-triangle tiles of the
// trailing block [k1, n), X = panel rows k0..k0+K-1, Y[2s] = X[2s+1],
// Y[2s+1] = -X[2s] (the FP64 mode's trailing update).
//
// Real FP64 on the FP64 tensor cores (dmma.cuh): one
// 128 x 128 upper tile per 512-thread block, each of the 16 warps a 32 x 32
// block of m8n8k4 fragments.  The C tile is loaded straight into the accumulators
// first, so its latency overlaps the copies of the panel rows; the panel rows
// arrive by cp.async in groups of 16 and each group is multiplied as soon as
// it lands.  A diagonal tile reads its Y rows from its own X rows.
constexpr int kDmmaBM = 128;
constexpr int kDmmaLD = kDmmaBM + 4;   // row stride in shared memory (4 mod 16 doubles)
constexpr int kDmmaThreads = 512;

template <int KMAX>
__global__ void __launch_bounds__(kDmmaThreads, 1)
gemm_dmma_kernel(double *__restrict__ W_all, int n, int k0, int K, const MatState *__restrict__ st_all)
{
    constexpr int GR = 16;                 // panel rows per copy group
    constexpr int NG = KMAX / GR;
    static_assert(KMAX % GR == 0 && NG <= 4, "copy groups");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Xs = reinterpret_cast<double *>(smem_raw);   // [KMAX][kDmmaLD]: rows k0.., columns a0..
    double *Ys = Xs + KMAX * kDmmaLD;                     // [KMAX][kDmmaLD]: rows k0.., columns b0..
    const int64_t b = blockIdx.x;
    if (st_all[b].dead) return;
    double *W = W_all + b * (int64_t)n * n;
    const int k1 = k0 + K;
    const int nt = (n - k1 + kDmmaBM - 1) / kDmmaBM;
    int I, J;
    upper_block(nt * (nt + 1) / 2 - 1 - (int)blockIdx.y, nt, I, J);
    const int a0 = k1 + I * kDmmaBM, b0 = k1 + J * kDmmaBM;
    const bool diag = I == J;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int wa = (warp >> 2) * 32, wb = (warp & 3) * 32;   // this warp's block in the tile

    double acc[4][4][2];
    load_c_frags<4, 4>(acc, W, n, a0 + wa, b0 + wb);

    constexpr int CPR = kDmmaBM / 2;       // 16-byte chunks per tile row
    const int per_group = GR * CPR * (diag ? 1 : 2);
#pragma unroll
    for (int gi = 0; gi < NG; gi++) {
        for (int e = tid; e < per_group; e += kDmmaThreads) {
            const int side = e >= GR * CPR;              // 0: X (columns a0..), 1: Y (columns b0..)
            const int e2 = side ? e - GR * CPR : e;
            const int r = gi * GR + e2 / CPR, c = 2 * (e2 % CPR);
            const int col = (side ? b0 : a0) + c;
            const bool ok = r < K && col < n;
            cp_async16((side ? Ys : Xs) + r * kDmmaLD + c, ok ? W + (int64_t)(k0 + r) * n + col : W, ok);
        }
        cp_async_commit();
    }
    const double *Yr = diag ? Xs : Ys;
    static_for<0, NG, 1>([&](auto gc) {
        constexpr int gi = decltype(gc)::value;
        cp_async_wait<NG - 1 - gi>();
        __syncthreads();
#pragma unroll 1
        for (int kb = gi * GR; kb < gi * GR + GR; kb += 4)
            dmma_kstep<4, 4>(acc, Xs + kb * kDmmaLD + wa, Yr + kb * kDmmaLD + wb, kDmmaLD);
    });
    store_c_frags<4, 4>(acc, W, n, a0 + wa, b0 + wb);
}

// The complex128 form: one 64 x 64 upper tile per 256-thread block, each warp
// a 32 x 16 block, four real m8n8k4 products per complex product (dmma.cuh);
// otherwise as gemm_dmma_kernel.
constexpr int kZdmmaBM = 64;
constexpr int kZdmmaLD = kZdmmaBM + 2;   // row stride in shared memory (2 mod 8 complex elements)

template <int KMAX>
__global__ void __launch_bounds__(256, 2)
gemm_zdmma_kernel(c128 *__restrict__ W_all, int n, int k0, int K, const MatState *__restrict__ st_all)
{
    constexpr int GR = 16;                 // panel rows per copy group
    constexpr int NG = KMAX / GR;
    static_assert(KMAX % GR == 0 && NG <= 4, "copy groups");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c128 *Xs = reinterpret_cast<c128 *>(smem_raw);   // [KMAX][kZdmmaLD]: rows k0.., columns a0..
    c128 *Ys = Xs + KMAX * kZdmmaLD;                  // [KMAX][kZdmmaLD]: rows k0.., columns b0..
    const int64_t b = blockIdx.x;
    if (st_all[b].dead) return;
    c128 *W = W_all + b * (int64_t)n * n;
    const int k1 = k0 + K;
    const int nt = (n - k1 + kZdmmaBM - 1) / kZdmmaBM;
    int I, J;
    upper_block(nt * (nt + 1) / 2 - 1 - (int)blockIdx.y, nt, I, J);
    const int a0 = k1 + I * kZdmmaBM, b0 = k1 + J * kZdmmaBM;
    const bool diag = I == J;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int wa = (warp >> 2) * 32, wb = (warp & 3) * 16;   // this warp's block in the tile

    double cr[4][2][2], ci[4][2][2];
    load_c_frags<4, 2>(cr, ci, W, n, a0 + wa, b0 + wb);

    const int per_group = GR * kZdmmaBM * (diag ? 1 : 2);   // 16-byte elements
#pragma unroll
    for (int gi = 0; gi < NG; gi++) {
        for (int e = tid; e < per_group; e += 256) {
            const int side = e >= GR * kZdmmaBM;
            const int e2 = side ? e - GR * kZdmmaBM : e;
            const int r = gi * GR + e2 / kZdmmaBM, c = e2 % kZdmmaBM;
            const int col = (side ? b0 : a0) + c;
            const bool ok = r < K && col < n;
            cp_async16((side ? Ys : Xs) + r * kZdmmaLD + c, ok ? W + (int64_t)(k0 + r) * n + col : W, ok);
        }
        cp_async_commit();
    }
    const c128 *Yr = diag ? Xs : Ys;
    static_for<0, NG, 1>([&](auto gc) {
        constexpr int gi = decltype(gc)::value;
        cp_async_wait<NG - 1 - gi>();
        __syncthreads();
#pragma unroll 1
        for (int kb = gi * GR; kb < gi * GR + GR; kb += 4)
            zdmma_kstep<4, 2, true>(cr, ci, Xs + kb * kZdmmaLD + wa, Yr + kb * kZdmmaLD + wb, kZdmmaLD);
    });
    store_c_frags<4, 2>(cr, ci, W, n, a0 + wa, b0 + wb);
}

// ----------------------------------------------------------------- finalize

// A device-side timeout of the update kernel (err != 0) yields log = NaN.
template <typename T>
__global__ void finalize_kernel(const MatState *__restrict__ st, const int32_t *__restrict__ err,
                                int64_t batch, int negate, double *__restrict__ log_out,
                                T *__restrict__ sign_out)
{
    const int64_t bidx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (bidx >= batch) return;
    const MatState s = st[bidx];
    if (err && err[bidx]) {
        log_out[bidx] = NAN;
        sign_out[bidx] = zero<T>();
        return;
    }
    if (s.dead) {
        log_out[bidx] = -INFINITY;
        sign_out[bidx] = zero<T>();
        return;
    }
    const double f = ((s.parity ^ negate) & 1) ? -1.0 : 1.0;
    log_out[bidx] = s.log_abs;
    if constexpr (IsComplex<T>::value) {
        using R = typename RealOf<T>::type;
        sign_out[bidx] = mk((R)(f * s.ph_re), (R)(f * s.ph_im));
    } else {
        sign_out[bidx] = (T)(f * s.ph_re);
    }
}

// ----------------------------------------------------------------- driver

template <typename T, int NB, int CPT>
// Matrices [b0, b0 + B) of a call on `batch` matrices, on stream s: the
// workspace is laid out for the whole call and this range uses its slices of
// it (A, log_out and sign_out are already offset to matrix b0).
static int run_large(const void *A, const void *const *Ap, int dtype, int64_t batch, int64_t b0, int64_t B, int n,
                     int layout, int mode, double *log_out, void *sign_out, unsigned char *ws, cudaStream_t s,
                     const pfb_slog_timing *tm, const pfb_slog_config &cf)
{
    const LargeLayout L = large_layout(dtype, batch, n, mode);
    int32_t *piv = reinterpret_cast<int32_t *>(ws + L.piv_off) + b0 * (n / 2);
    MatState *st = reinterpret_cast<MatState *>(ws + L.st_off) + b0;
    T *W = reinterpret_cast<T *>(ws + L.w_off) + b0 * (int64_t)n * n;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    {
        int64_t blocks = (B * (int64_t)n + 7) / 8;   // 8 warps (rows) per block
        if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
        if (blocks < 1) blocks = 1;
        switch (dtype) {
        case PFB_F32:
            copy_in_kernel<float, double><<<(unsigned)blocks, 256, 0, s>>>((const float *)A, (const float *const *)Ap, (double *)W, B, n, st);
            break;
        case PFB_F64:
            copy_in_kernel<double, double><<<(unsigned)blocks, 256, 0, s>>>((const double *)A, (const double *const *)Ap, (double *)W, B, n, st);
            break;
        case PFB_C64:
            copy_in_kernel<c64, c128><<<(unsigned)blocks, 256, 0, s>>>((const c64 *)A, (const c64 *const *)Ap, (c128 *)W, B, n, st);
            break;
        default:
            copy_in_kernel<c128, c128><<<(unsigned)blocks, 256, 0, s>>>((const c128 *)A, (const c128 *const *)Ap, (c128 *)W, B, n, st);
            break;
        }
        if (launch_status() != PFB_OK) return PFB_ERR_CUDA;
    }

    // the panel form: the whole window in registers (one CTA per SM), or half
    // of it in shared memory (two CTAs per SM; one trailing column per thread)
    void (*pk)(T *, int, int, MatState *, int32_t *) = panel_kernel<T, NB, CPT>;
    size_t psmem = sizeof(PanelSmem<T, NB>);
    if constexpr (CPT == 1) {
        if (cf.panel == PFB_PANEL_HALF_SHARED) {
            pk = panel_hs_kernel<T, NB>;
            psmem = sizeof(PanelSmemHS<T, NB>);
        }
    }
    if (cuda_check(cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem)) != PFB_OK) return PFB_ERR_CUDA;
    if (cuda_check(cudaFuncSetAttribute(pk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != PFB_OK) return PFB_ERR_CUDA;

    constexpr bool cplx = IsComplex<T>::value;
    // FP64 tensor-core tiles: 128 x 128 real, 64 x 64 complex
    constexpr int BM = cplx ? kZdmmaBM : kDmmaBM;
    void *gk;
    size_t gsmem;
    if constexpr (cplx) {
        gk = (void *)gemm_zdmma_kernel<NB>;
        gsmem = (size_t)2 * NB * kZdmmaLD * sizeof(c128);
    } else {
        gk = (void *)gemm_dmma_kernel<NB>;
        gsmem = (size_t)2 * NB * kDmmaLD * sizeof(double);
    }
    if (cuda_check(cudaFuncSetAttribute(gk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem)) != PFB_OK) return PFB_ERR_CUDA;

    SplitArgs sa{};
    unsigned char *split_ws = ws + L.split_off;
    const int slices = cf.slices;
    int32_t *split_err = nullptr;
    if ((mode & 0xff) == PFB_MODE_SPLIT) {
        split_err = split_args(true, split_ws, cplx, batch, n, NB, 0, slices).err + b0;
        if (cuda_check(cudaMemsetAsync(split_err, 0, (size_t)B * sizeof(int32_t), s)) != PFB_OK) return PFB_ERR_CUDA;
    }
    auto rec = [&](void **evs, int i) {
        if (tm && evs && i < 2 * tm->pairs) cudaEventRecord((cudaEvent_t)evs[i], s);
    };
    int panel_idx = 0;
    for (int k0 = 0; k0 < n - 1; k0 += NB, panel_idx++) {
        const int K = (n - k0 < NB) ? n - k0 : NB;
        const int mt = n - (k0 + NB);
        int CL = mt > 0 ? (mt + kTT * CPT - 1) / (kTT * CPT) : 1;
        if (CL < 1) CL = 1;
        if (CL > kClusterMax) return PFB_ERR_SIZE;
        const bool use_split = (mode & 0xff) == PFB_MODE_SPLIT && mt > 0;
        sa = split_args(use_split, split_ws, cplx, batch, n, NB, k0, slices);
        sa.epilogue = cf.epilogue;
        if (mode & PFB_SPLIT_TEST_TIMEOUT) sa.fail_b = 0;
        sa = split_shift(sa, b0);

        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)CL, (unsigned)B, 1);
        cfg.blockDim = dim3(kTT, 1, 1);
        cfg.dynamicSmemBytes = psmem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)CL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        rec(tm ? tm->panel_events : nullptr, 2 * panel_idx);
        if (cuda_check(cudaLaunchKernelEx(&cfg, pk, W, n, k0, st, piv)) != PFB_OK) return PFB_ERR_CUDA;
        rec(tm ? tm->panel_events : nullptr, 2 * panel_idx + 1);

        if (mt > 0) {
            rec(tm ? tm->update_events : nullptr, 2 * panel_idx);
            if (use_split) {
                constexpr int cpb = 256 / (NB / 16);
                split_slice_kernel<T, NB><<<dim3((unsigned)((mt + cpb - 1) / cpb), (unsigned)B), 256, 0, s>>>(
                    W, n, k0, st, sa);
                if (launch_status() != PFB_OK) return PFB_ERR_CUDA;
                int rc = launch_split_update(cplx, W, n, k0, K, B, st, sa, s);
                if (rc != PFB_OK) return rc;
            } else {
                const int nt = (mt + BM - 1) / BM;
                const unsigned tiles = (unsigned)(nt * (nt + 1) / 2);
                // blockIdx.x = matrix, blockIdx.y = tile from the last: the blocks start in
                // that order, so the first row tile (the next panel's rows) is written
                // last and is still in L2 when the next panel loads it
                if constexpr (cplx)
                    gemm_zdmma_kernel<NB><<<dim3((unsigned)B, tiles), 256, gsmem, s>>>(W, n, k0, K, st);
                else
                    gemm_dmma_kernel<NB><<<dim3((unsigned)B, tiles), kDmmaThreads, gsmem, s>>>(W, n, k0, K, st);
                if (launch_status() != PFB_OK) return PFB_ERR_CUDA;
            }
            rec(tm ? tm->update_events : nullptr, 2 * panel_idx + 1);
        }
    }

    const int negate = (layout == PFB_COL_MAJOR) ? ((n >> 1) & 1) : 0;
    const unsigned fb = (unsigned)((B + 127) / 128);
    switch (dtype) {
    case PFB_F32: finalize_kernel<float><<<fb, 128, 0, s>>>(st, split_err, B, negate, log_out, (float *)sign_out); break;
    case PFB_F64: finalize_kernel<double><<<fb, 128, 0, s>>>(st, split_err, B, negate, log_out, (double *)sign_out); break;
    case PFB_C64: finalize_kernel<c64><<<fb, 128, 0, s>>>(st, split_err, B, negate, log_out, (c64 *)sign_out); break;
    default: finalize_kernel<c128><<<fb, 128, 0, s>>>(st, split_err, B, negate, log_out, (c128 *)sign_out); break;
    }
    return launch_status();
}

template <typename T, int NB, int CPT>
static int max_concurrent_t(int n, int panel)
{
    const int mt = n - NB;
    int CL = mt > 0 ? (mt + kTT * CPT - 1) / (kTT * CPT) : 1;
    if (CL < 1) CL = 1;
    void (*pk)(T *, int, int, MatState *, int32_t *) = panel_kernel<T, NB, CPT>;
    size_t psmem = sizeof(PanelSmem<T, NB>);
    if constexpr (CPT == 1) {
        if (panel == PFB_PANEL_HALF_SHARED) {
            pk = panel_hs_kernel<T, NB>;
            psmem = sizeof(PanelSmemHS<T, NB>);
        }
    }
    if (cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem) != cudaSuccess) return 0;
    if (cudaFuncSetAttribute(pk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) return 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)CL, 1, 1);
    cfg.blockDim = dim3(kTT, 1, 1);
    cfg.dynamicSmemBytes = psmem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int num = 0;
    if (cudaOccupancyMaxActiveClusters(&num, (const void *)pk, &cfg) != cudaSuccess) return 0;
    return num;
}

int large_max_concurrent(int dtype, int n, int panel)
{
    int nb = 0, cpt = 0;
    if (!large_cfg(dtype, n, &nb, &cpt)) return 0;
    const bool cplx = dtype == PFB_C64 || dtype == PFB_C128;
    if (!cplx) return nb == 64 ? max_concurrent_t<double, 64, 1>(n, panel) : max_concurrent_t<double, 32, 2>(n, panel);
    return max_concurrent_t<c128, 32, 1>(n, panel);
}

// Whether the half-shared panel form exists for this order (one trailing
// column per thread).
static bool hs_available(int dtype, int n)
{
    int nb = 0, cpt = 0;
    return large_cfg(dtype, n, &nb, &cpt) && cpt == 1;
}

static int run_large_range(int dtype, const void *A, const void *const *Ap, int64_t batch, int64_t b0, int64_t B,
                           int n, int layout, int mode, double *log_out, void *sign_out, unsigned char *ws,
                           cudaStream_t s, const pfb_slog_timing *timing, const pfb_slog_config &cf)
{
    int nb = 0, cpt = 0;
    large_cfg(dtype, n, &nb, &cpt);
    const size_t in_es = dtype == PFB_F32 ? 4 : (dtype == PFB_C128 ? 16 : 8);
    const size_t sign_es = in_es;
    const void *a = Ap ? nullptr : static_cast<const char *>(A) + (size_t)b0 * (size_t)n * (size_t)n * in_es;
    const void *const *ap = Ap ? Ap + b0 : nullptr;
    double *lo = log_out + b0;
    void *so = static_cast<char *>(sign_out) + (size_t)b0 * sign_es;
    const bool cplx = dtype == PFB_C64 || dtype == PFB_C128;
    if (!cplx) {
        if (nb == 64)
            return run_large<double, 64, 1>(a, ap, dtype, batch, b0, B, n, layout, mode, lo, so, ws, s, timing, cf);
        return run_large<double, 32, 2>(a, ap, dtype, batch, b0, B, n, layout, mode, lo, so, ws, s, timing, cf);
    }
    return run_large<c128, 32, 1>(a, ap, dtype, batch, b0, B, n, layout, mode, lo, so, ws, s, timing, cf);
}

// The second stream of this host thread's calls on device `dev`: one per thread
// and device, created on first use and destroyed when the thread exits.  Per
// thread, so that callers on other threads never share it: their calls stay
// independent, and a graph capture on one thread cannot pull in another
// thread's work.
struct AuxStreams {
    cudaStream_t s[64] = {};
    ~AuxStreams()
    {
        for (cudaStream_t x : s)
            if (x) cudaStreamDestroy(x);
    }
};

static cudaStream_t aux_stream(int dev)
{
    thread_local AuxStreams aux;
    if (dev < 0 || dev >= 64) return nullptr;
    if (!aux.s[dev] && cudaStreamCreateWithFlags(&aux.s[dev], cudaStreamNonBlocking) != cudaSuccess)
        aux.s[dev] = nullptr;
    return aux.s[dev];
}

// Whether work forked from `caller` onto `aux` stays in the caller's own
// capture state: a stream that joined a graph capture belongs to it until that
// capture ends, so while `aux` is part of a capture, only a call on a stream of
// that same capture may use it.
static bool aux_usable(cudaStream_t caller, cudaStream_t aux)
{
    cudaStreamCaptureStatus ca = cudaStreamCaptureStatusNone, cc = cudaStreamCaptureStatusNone;
    unsigned long long ia = 0, ic = 0;
    if (cudaStreamGetCaptureInfo(aux, &ca, &ia) != cudaSuccess) return false;
    if (ca == cudaStreamCaptureStatusNone) return true;
    if (cudaStreamGetCaptureInfo(caller, &cc, &ic) != cudaSuccess) return false;
    return ca == cudaStreamCaptureStatusActive && cc == cudaStreamCaptureStatusActive && ia == ic;
}

// A batch of three or more waves of the widest panel clusters (clusters of 9
// or more CTAs: one per GPC, so the panel waves leave SMs idle) is run as two
// ranges on two streams, the last wave's worth of matrices on the second: its
// updates fill the SMs the first range's panel waves leave idle (2n = 4096,
// batch 28: 43.0 -> 41.9 ms).  The second stream forks from and joins the
// caller's stream through events, so the call stays ordered on `stream` and
// can be captured in a CUDA graph.  The second stream is this host thread's own
// (aux_stream); when it is part of another capture the call runs as one range.
//
// The configuration of a call: the caller's fields where it gives them, else
// the tuned table's choice for (dtype, n, batch) (tune_table.h, written by
// pfcuda_b200/tune.py), else the defaults.  Returns false for an invalid
// override.
bool large_config(int dtype, int64_t batch, int n, int mode, const pfb_slog_config *over, pfb_slog_config *out)
{
    pfb_slog_config c = tuned_config(dtype, n, batch, (mode & 0xff) == PFB_MODE_SPLIT);
    if (!hs_available(dtype, n)) c.panel = PFB_PANEL_REGISTERS;
    if ((mode >> 8) & 0xf) c.slices = (mode >> 8) & 0xf;
    if (over) {
        if (over->panel < 0 || over->panel > 2 || over->slices < 0 || over->slices > kSplitMaxSlices ||
            over->ranges < 0 || over->ranges > 2 || over->epilogue < 0 || over->epilogue > 3)
            return false;
        if (over->panel) {
            if (over->panel == PFB_PANEL_HALF_SHARED && !hs_available(dtype, n)) return false;
            c.panel = over->panel;
        }
        if (over->slices) c.slices = over->slices;
        if (over->ranges) c.ranges = over->ranges;
        if (over->epilogue) c.epilogue = over->epilogue;
    }
    *out = c;
    return true;
}

// The size of the second range (0: one range) for a call on `batch` matrices,
// when the configuration asks for two ranges and the widest panel clusters
// have 9 or more CTAs: the last wave's worth of them for a batch of three waves
// or more, half the batch for a batch of two waves or more.
int64_t large_second_range(int dtype, int64_t batch, int n, const pfb_slog_config &cf)
{
    int nb = 0, cpt = 0;
    if (cf.ranges != 2 || !large_cfg(dtype, n, &nb, &cpt)) return 0;
    const int widest = (n - nb + kTT * cpt - 1) / (kTT * cpt);
    if (widest < 9) return 0;
    const int64_t mc = large_max_concurrent(dtype, n, cf.panel);
    if (mc <= 0) return 0;
    if (batch >= 3 * mc) return mc;
    if (batch >= 2 * mc) return batch / 2;
    return 0;
}

int launch_large(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                 double *log_out, void *sign_out, void *workspace, size_t workspace_bytes,
                 cudaStream_t stream, const pfb_slog_timing *timing, const pfb_slog_config *over,
                 const void *const *A_ptrs)
{
    int nb = 0, cpt = 0;
    if (!large_cfg(dtype, n, &nb, &cpt)) return PFB_ERR_SIZE;
    if ((mode & 0xff) == PFB_MODE_SPLIT && !split_available()) return PFB_ERR_UNSUPPORTED;
    if (batch > 65535) return PFB_ERR_SIZE;
    pfb_slog_config cf;
    if (!large_config(dtype, batch, n, mode, over, &cf)) return PFB_ERR_INVALID;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    const int64_t mc = timing == nullptr ? large_second_range(dtype, batch, n, cf) : 0;
    int dev = 0;
    cudaStream_t s2 = nullptr;
    if (mc > 0 && cudaGetDevice(&dev) == cudaSuccess) s2 = aux_stream(dev);
    if (s2 && !aux_usable(stream, s2)) s2 = nullptr;
    if (!s2)
        return run_large_range(dtype, A, A_ptrs, batch, 0, batch, n, layout, mode, log_out, sign_out, ws, stream,
                               timing, cf);

    const int64_t B2 = mc, B1 = batch - B2;
    cudaEvent_t fork, join;
    if (cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess) return PFB_ERR_CUDA;
    if (cudaEventCreateWithFlags(&join, cudaEventDisableTiming) != cudaSuccess) {
        cudaEventDestroy(fork);
        return PFB_ERR_CUDA;
    }
    int rc = PFB_OK;
    if (cudaEventRecord(fork, stream) != cudaSuccess || cudaStreamWaitEvent(s2, fork, 0) != cudaSuccess)
        rc = PFB_ERR_CUDA;
    if (rc == PFB_OK)
        rc = run_large_range(dtype, A, A_ptrs, batch, 0, B1, n, layout, mode, log_out, sign_out, ws, stream, nullptr,
                             cf);
    // the second range always runs (or at least joins), so the fork is always closed
    const int rc2 = rc == PFB_OK ? run_large_range(dtype, A, A_ptrs, batch, B1, B2, n, layout, mode, log_out,
                                                   sign_out, ws, s2, nullptr, cf)
                                 : PFB_OK;
    if (cudaEventRecord(join, s2) != cudaSuccess || cudaStreamWaitEvent(stream, join, 0) != cudaSuccess)
        rc = PFB_ERR_CUDA;
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    return rc != PFB_OK ? rc : rc2;
}

int large_copy_pivots(int64_t batch, int n, const void *workspace, size_t workspace_bytes,
                      int32_t *piv_out, cudaStream_t stream)
{
    const size_t bytes = (size_t)batch * (size_t)(n / 2) * sizeof(int32_t);
    if (workspace_bytes < bytes) return PFB_ERR_WORKSPACE;
    return cudaMemcpyAsync(piv_out, workspace, bytes, cudaMemcpyDeviceToDevice, stream) == cudaSuccess
               ? PFB_OK
               : PFB_ERR_CUDA;
}

}  // namespace pfb
