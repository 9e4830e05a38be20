// split.cu -- split-precision trailing update of the blocked factorisation on
// the tcgen05 tensor cores.
//
// The update S22 += X^T Y (large.cu) has an inner dimension of only one panel
// (K = 64 real, 2 x 32 complex).  Each factor is split without error into int8
// digits (Ozaki, Ogita, Oishi and Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 2012; the integer variant of Ootomo, Ozaki
// and Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 2024):
//
//   x_a[k] = 2^e_a * sum_{i<S} 2^(-7(i+1)) X_i[a][k],   X_i in [-127, 127]
//
// with one power-of-two scale per trailing index a (split.cuh, written by the
// panel kernel).  Then
//
//   sum_k x_a[k] y_b[k] ~= 2^(e_a+e_b) sum_{l<S} 2^(-7(l+2)) P_l[a][b],
//   P_l = sum_{i+j=l} X_i Y_j^T
//
// and every P_l is an exact int32 sum (|P_l| <= S * K * 127^2 < 2^31), formed by
// tcgen05.mma.kind::i8 into its own TMEM accumulator.  The epilogue converts
// the S accumulators to FP64, recombines them (smallest level first) and adds
// the result to the FP64 working matrix.  Dropped terms are those with
// i + j >= S and the digits beyond S, a relative error of about K * 2^(-7S) of
// |x_a| |y_b|.
//
// Kernel shape (one CTA per output tile, 128 threads):
//   * the A chunk (128 trailing rows) and B chunk (TN rows) of every slice are
//     the exact shared-memory images of the MMA operands (split.cuh), fetched by
//     one thread with bulk asynchronous copies (cp.async.bulk, the TMA engine)
//     completing on an mbarrier;
//   * one thread issues all S(S+1)/2 * K/32 MMAs of the tile into S TMEM
//     accumulators (TN columns each), then commits to a second mbarrier;
//   * the four warps read their 32 TMEM lanes (rows) back with tcgen05.ld and
//     update the FP64 tile.
// Every mbarrier wait is bounded; a wait that gives up marks the matrix in
// SplitArgs::err and the kernel frees its TMEM and returns.
#include <stdio.h>

#include "split.cuh"
#include "large.cuh"

namespace pfb {

constexpr int kSplitThreads = 128;
constexpr long long kWaitSpins = 1LL << 24;   // bounded mbarrier polling

bool split_available()
{
    int dev = 0, major = 0, minor = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    return major == 10 && minor == 0;
}

static int split_kk(bool cplx, int nb) { return cplx ? 2 * nb : nb; }

size_t split_workspace_bytes(bool cplx, int64_t batch, int n, int nb)
{
    const int kk = split_kk(cplx, nb);
    const int ntile = (n + kSplitTileM - 1) / kSplitTileM;
    const size_t per = (size_t)kSplitMaxSlices * ntile * kSplitTileM * kk;
    const size_t arrays = cplx ? 3 : 2;
    return (size_t)batch * (arrays * per + (size_t)n * 4 + 4) + 4096;
}

SplitArgs split_args(bool use, unsigned char *ws, bool cplx, int64_t batch, int n, int nb, int k0,
                     int slices)
{
    SplitArgs a{};
    a.enabled = use ? 1 : 0;
    a.n = n;
    a.k0 = k0;
    a.nb = nb;
    a.kk = split_kk(cplx, nb);
    a.slices = slices;
    a.cplx = cplx ? 1 : 0;
    a.ntile = (n + kSplitTileM - 1) / kSplitTileM;
    a.mstride = (int64_t)kSplitMaxSlices * a.ntile * kSplitTileM * a.kk;
    a.xs = reinterpret_cast<int8_t *>(ws);
    a.ys = a.xs + batch * a.mstride;
    a.ys2 = cplx ? a.ys + batch * a.mstride : nullptr;
    int8_t *end = (cplx ? a.ys2 : a.ys) + batch * a.mstride;
    a.ex = reinterpret_cast<int32_t *>(end);
    a.err = a.ex + batch * (int64_t)n;
    return a;
}

// ------------------------------------------------------------- PTX wrappers

PFB_D uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

PFB_D void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
PFB_D void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
PFB_D bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
PFB_D bool mbar_wait_bounded(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kWaitSpins; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
PFB_D void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}
PFB_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
PFB_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

PFB_D uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    // K-major, no swizzle: start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46),
    // version 1 at [46,48), base offset 0, layout type 0 (SWIZZLE_NONE) at [61,64)
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor of kind::i8: D = S32 [4,6), A = B = signed int8
// [7,10) / [10,13), both K-major, N>>3 at [17,23), M>>4 at [24,29)
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

PFB_D void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}
PFB_D void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(bar) : "memory");
}
PFB_D void tmem_ld16(uint32_t taddr, int32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                 : "r"(taddr));
}
PFB_D void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ------------------------------------------------------------------ kernel

// One (128 x TN) tile of the upper triangle of the trailing block per CTA.
// NOUT = 1 (real) or 2 (complex: real and imaginary parts from B1, B2).
template <int TN, int NOUT>
__global__ void __launch_bounds__(kSplitThreads, 1)
split_update_kernel(void *__restrict__ W_all, int n, int k0, int K, MatState *__restrict__ st_all,
                    SplitArgs sa)
{
    constexpr int TM = kSplitTileM;
    constexpr uint32_t TMEM_COLS = 512;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int kk = sa.kk;                        // bytes per operand row (K of the int8 products)
    const int S = sa.slices;
    const int a_bytes = TM * kk;                 // one slice of the A tile
    const int b_bytes = TN * kk;                 // one slice of one B tile
    unsigned char *sA = smem;
    unsigned char *sB = sA + kSplitMaxSlices * a_bytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + NOUT * kSplitMaxSlices * b_bytes);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
    int *s_ex = reinterpret_cast<int *>(tmem_slot + 4);          // TN exponents of the B rows
    int *s_flag = s_ex + TN;

    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    const int k1 = k0 + K;
    const int m = n - k1;
    const int ntn = (m + TN - 1) / TN;
    // upper-triangle tiles: row tile I (TM rows) needs column tiles J with
    // TN*(J+1) > TM*I, i.e. J >= I*TM/TN
    constexpr int R = TM / TN;
    const int ntm = (m + TM - 1) / TM;
    int L = blockIdx.x, I = 0;
    while (I < ntm && L >= ntn - I * R) { L -= ntn - I * R; I++; }
    if (I >= ntm) return;
    const int J = I * R + L;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    const uint32_t bar_ld = su32(&bars[0]), bar_mma = su32(&bars[1]);
    if (tid == 0) {
        mbar_init(bar_ld, 1);
        mbar_init(bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *s_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(su32(tmem_slot)), "r"(TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid < TN) {
        const int col = k1 + J * TN + tid;
        s_ex[tid] = col < n ? sa.ex[b * n + col] : 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // ---- operands: S slices of the A tile and of the B tile(s), one mbarrier
    if (tid == 0) {
        const uint32_t total = (uint32_t)S * (a_bytes + NOUT * b_bytes);
        mbar_expect_tx(bar_ld, total);
        const int64_t chunk = (int64_t)TM * kk;
        const int jrow = J * TN;                                  // first B row
        const int64_t boff = (int64_t)(jrow / TM) * chunk + (int64_t)((jrow % TM) >> 3) * (kk >> 4) * 128;
        for (int s = 0; s < S; s++) {
            const int8_t *ga = sa.xs + b * sa.mstride + ((int64_t)s * sa.ntile + I) * chunk;
            bulk_g2s(su32(sA + s * a_bytes), ga, a_bytes, bar_ld);
            const int8_t *gb = sa.ys + b * sa.mstride + (int64_t)s * sa.ntile * chunk + boff;
            bulk_g2s(su32(sB + s * b_bytes), gb, b_bytes, bar_ld);
            if (NOUT == 2) {
                const int8_t *gb2 = sa.ys2 + b * sa.mstride + (int64_t)s * sa.ntile * chunk + boff;
                bulk_g2s(su32(sB + (kSplitMaxSlices + s) * b_bytes), gb2, b_bytes, bar_ld);
            }
        }
    }
    bool ok = mbar_wait_bounded(bar_ld, 0);

    // ---- MMAs: level l accumulates sum_{i+j=l} A_i B_j^T in TMEM columns [l*TN, (l+1)*TN)
    if (tid == 0) {
        if (ok) {
            tc_fence_after();
            constexpr uint32_t idesc = idesc_i8(TM, TN);
            const uint32_t sbo = (uint32_t)(kk >> 4) * 128;     // next 8-row group
            for (int o = 0; o < NOUT; o++) {
                for (int l = 0; l < S; l++) {
                    const uint32_t dcol = (uint32_t)((o * S + l) * TN);
                    for (int i = 0; i <= l; i++) {
                        const int j = l - i;
                        for (int kc = 0; kc < kk / 32; kc++) {
                            const uint64_t ad = smem_desc(su32(sA + i * a_bytes + kc * 256), 128, sbo);
                            const uint64_t bd = smem_desc(su32(sB + (o * kSplitMaxSlices + j) * b_bytes + kc * 256), 128, sbo);
                            mma_i8(tmem + dcol, ad, bd, idesc, (i > 0 || kc > 0) ? 1u : 0u);
                        }
                    }
                }
            }
            mma_commit(bar_mma);
        } else {
            *s_flag = 1;
        }
    }
    __syncthreads();
    if (*s_flag) ok = false;
    if (ok) ok = mbar_wait_bounded(bar_mma, 0);
    tc_fence_after();

    // ---- epilogue: thread = tile row; combine the S levels in FP64 and add to W
    const int arow = k1 + I * TM + warp * 32 + lane;
    if (ok) {
        const int ea = arow < n ? sa.ex[b * n + arow] : 0;
        for (int cb = 0; cb < TN / 16; cb++) {
            double vr[NOUT][16];
#pragma unroll
            for (int o = 0; o < NOUT; o++)
#pragma unroll
                for (int c = 0; c < 16; c++) vr[o][c] = 0.0;
            for (int o = 0; o < NOUT; o++) {
                for (int l = S - 1; l >= 0; l--) {         // smallest contributions first
                    int32_t v[16];
                    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) +
                                           (uint32_t)((o * S + l) * TN + cb * 16);
                    tmem_ld16(taddr, v);
                    tmem_ld_wait();
                    const double sc = ldexp(1.0, -7 * (l + 2));
#pragma unroll
                    for (int c = 0; c < 16; c++) vr[o][c] = fma((double)v[c], sc, vr[o][c]);
                }
            }
            if (arow < n) {
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    const int bcol = k1 + J * TN + cb * 16 + c;
                    if (bcol < n && bcol > arow) {
                        const int e = ea + s_ex[cb * 16 + c];
                        if (NOUT == 1) {
                            double *p = reinterpret_cast<double *>(W_all) + b * (int64_t)n * n + (int64_t)arow * n + bcol;
                            *p += ldexp(vr[0][c], e);
                        } else {
                            double *p = reinterpret_cast<double *>(W_all) + 2 * (b * (int64_t)n * n + (int64_t)arow * n + bcol);
                            p[0] += ldexp(vr[0][c], e);
                            p[1] += ldexp(vr[NOUT - 1][c], e);
                        }
                    }
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(&sa.err[b], PFB_ERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// At least 120 KB so that one CTA (holding all 512 TMEM columns) runs per SM.
template <int TN, int NOUT>
static size_t split_smem_bytes(int kk)
{
    const size_t need = (size_t)kSplitMaxSlices * kSplitTileM * kk + (size_t)NOUT * kSplitMaxSlices * TN * kk +
                        64 + TN * sizeof(int) + 16;
    return need < 120 * 1024 ? 120 * 1024 : need;
}

int launch_split_update(bool cplx, void *W, int n, int k0, int K, int64_t batch, MatState *st,
                        const SplitArgs &sa, cudaStream_t stream)
{
    const int k1 = k0 + K;
    const int m = n - k1;
    if (m <= 0) return PFB_OK;
    if (!cplx) {
        constexpr int TN = 64;
        const int ntn = (m + TN - 1) / TN;
        const int ntm = (m + kSplitTileM - 1) / kSplitTileM;
        int tiles = 0;
        for (int I = 0; I < ntm; I++) tiles += ntn - I * (kSplitTileM / TN) > 0 ? ntn - I * (kSplitTileM / TN) : 0;
        auto k = split_update_kernel<TN, 1>;
        const size_t smem = split_smem_bytes<TN, 1>(sa.kk);
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return PFB_ERR_CUDA;
        k<<<dim3((unsigned)tiles, (unsigned)batch), kSplitThreads, smem, stream>>>(W, n, k0, K, st, sa);
    } else {
        constexpr int TN = 32;
        const int ntn = (m + TN - 1) / TN;
        const int ntm = (m + kSplitTileM - 1) / kSplitTileM;
        int tiles = 0;
        for (int I = 0; I < ntm; I++) tiles += ntn - I * (kSplitTileM / TN) > 0 ? ntn - I * (kSplitTileM / TN) : 0;
        auto k = split_update_kernel<TN, 2>;
        const size_t smem = split_smem_bytes<TN, 2>(sa.kk);
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return PFB_ERR_CUDA;
        k<<<dim3((unsigned)tiles, (unsigned)batch), kSplitThreads, smem, stream>>>(W, n, k0, K, st, sa);
    }
    return cudaGetLastError() == cudaSuccess ? PFB_OK : PFB_ERR_CUDA;
}

}  // namespace pfb
