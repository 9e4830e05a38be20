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
// The A chunk (128 trailing rows) and B chunk (TN rows) of every slice are the
// exact shared-memory images of the MMA operands (split.cuh), fetched with bulk
// asynchronous copies (cp.async.bulk, the TMA engine) completing on mbarriers;
// one thread issues the S(S+1)/2 * K/32 MMAs of a tile into S TMEM accumulators
// of TN columns; the epilogue warps read their TMEM lanes back with tcgen05.ld.
// Every mbarrier wait is bounded; a wait that gives up marks the matrix in
// SplitArgs::err and the kernel frees its TMEM and returns.
#include <stdio.h>

#include "split.cuh"
#include "large.cuh"

namespace pfb {

constexpr int kSplitThreads = 320;   // warp 0: loads, warp 1: MMA, warps 2-9: epilogue
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

PFB_D void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
PFB_D void tmem_ld8(uint32_t taddr, int32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

// Upper-triangle tiles of the trailing block in row-major order: row tile I
// (TM rows) holds column tiles J = I*R .. ntn-1, R = TM/TN.
struct TileWalk {
    int ntn, R, I, J;
    PFB_D void start(int idx)
    {
        I = 0;
        while (idx >= ntn - I * R) { idx -= ntn - I * R; I++; }
        J = I * R + idx;
    }
    PFB_D void next()
    {
        if (++J >= ntn) { I++; J = I * R; }
    }
};

// Persistent, warp-specialised update of the upper-triangle (128 x TN) tiles
// of one matrix's trailing block (blockIdx.y = matrix, blockIdx.x = CTA):
//   warp 0   bulk copies of the operand chunks (the TMA engine),
//   warp 1   one thread issues the tcgen05 MMAs,
//   warps 2-9  epilogue: warp w reads TMEM lane quarter w%4 (the only one it
//            may access) and the half h = (w-2)/4 of the tile's columns.
// Each CTA walks a contiguous range of tiles, so consecutive tiles mostly share
// the A operand (the 128 trailing rows), which stays in shared memory; the B
// operands rotate through two stages.  The S digit-level accumulators of a tile
// (NOUT * S * TN <= 448 TMEM columns) are handed back to the MMA thread as soon
// as the epilogue has read them, so the next tile's MMAs overlap this tile's
// FP64 read-modify-write of W, and the C values of the next tile are loaded
// while its MMAs run.
//
// Epilogue arithmetic: |P_l| < 2^23 (at most 7 * 64 products of 127^2), so
//   hi = sum_{l<=3} P_l * 2^(7(3-l)),  lo = sum_{l>=4} P_l * 2^(7(6-l))
// are exact integers below 2^53, and the tile value is
//   2^(e_a+e_b) * (hi * 2^-35 + lo * 2^-56)
// with a single rounding.
template <int TN, int NOUT>
__global__ void __launch_bounds__(kSplitThreads, 1)
split_update_kernel(void *__restrict__ W_all, int n, int k0, int K, MatState *__restrict__ st_all,
                    SplitArgs sa)
{
    constexpr int TM = kSplitTileM;
    constexpr uint32_t TMEM_COLS = 512;
    constexpr int CW = TN / 2;                  // columns per epilogue thread
    constexpr int NV = CW * NOUT / 2;           // double2 vectors of W per thread and tile
    extern __shared__ __align__(1024) unsigned char smem[];
    const int kk = sa.kk;
    const int S = sa.slices;
    const int a_bytes = TM * kk;                // one slice of the A tile
    const int b_bytes = TN * kk;                // one slice of one B tile
    const int bstage = NOUT * kSplitMaxSlices * b_bytes;
    unsigned char *sA = smem;
    unsigned char *sB = sA + kSplitMaxSlices * a_bytes;     // two stages
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + 2 * bstage);
    // bars: 0 a_full, 1 a_empty, 2-3 b_full, 4-5 b_empty, 6 acc_full, 7 acc_empty
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 8);
    int *s_fail = reinterpret_cast<int *>(tmem_slot + 1);

    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    const int k1 = k0 + K;
    const int m = n - k1;
    const int ntn = (m + TN - 1) / TN;
    const int ntm = (m + TM - 1) / TM;
    constexpr int R = TM / TN;
    int total = 0;
    for (int I = 0; I < ntm; I++) total += ntn - I * R > 0 ? ntn - I * R : 0;
    const int t0 = (int)((int64_t)total * blockIdx.x / gridDim.x);
    const int t1 = (int)((int64_t)total * (blockIdx.x + 1) / gridDim.x);
    if (t0 >= t1) return;
    const int ntiles = t1 - t0;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t bar[8];
#pragma unroll
    for (int i = 0; i < 8; i++) bar[i] = su32(&bars[i]);
    if (tid == 0) {
        for (int i = 0; i < 7; i++) mbar_init(bar[i], 1);
        mbar_init(bar[7], 256);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *s_fail = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(su32(tmem_slot)), "r"(TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0) {
        // ---------------- producer
        if (lane == 0) {
            const int64_t chunk = (int64_t)TM * kk;
            TileWalk tw{ntn, R, 0, 0};
            tw.start(t0);
            int arow = -1, aloads = 0;
            for (int it = 0; it < ntiles && ok; it++, tw.next()) {
                if (tw.I != arow) {
                    if (aloads > 0) ok = mbar_wait_bounded(bar[1], (aloads - 1) & 1);
                    if (!ok) break;
                    mbar_expect_tx(bar[0], (uint32_t)(S * a_bytes));
                    for (int s = 0; s < S; s++)
                        bulk_g2s(su32(sA + s * a_bytes),
                                 sa.xs + b * sa.mstride + ((int64_t)s * sa.ntile + tw.I) * chunk, a_bytes, bar[0]);
                    arow = tw.I;
                    aloads++;
                }
                const int st = it & 1;
                if (it >= 2) ok = mbar_wait_bounded(bar[4 + st], ((it >> 1) - 1) & 1);
                if (!ok) break;
                const int jrow = tw.J * TN;
                const int64_t boff = (int64_t)(jrow / TM) * chunk + (int64_t)((jrow % TM) >> 3) * (kk >> 4) * 128;
                mbar_expect_tx(bar[2 + st], (uint32_t)(S * NOUT * b_bytes));
                unsigned char *dst = sB + st * bstage;
                for (int s = 0; s < S; s++) {
                    bulk_g2s(su32(dst + s * b_bytes), sa.ys + b * sa.mstride + (int64_t)s * sa.ntile * chunk + boff,
                             b_bytes, bar[2 + st]);
                    if (NOUT == 2)
                        bulk_g2s(su32(dst + (kSplitMaxSlices + s) * b_bytes),
                                 sa.ys2 + b * sa.mstride + (int64_t)s * sa.ntile * chunk + boff, b_bytes, bar[2 + st]);
                }
            }
            if (!ok) atomicExch(s_fail, 1);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_i8(TM, TN);
            const uint32_t sbo = (uint32_t)(kk >> 4) * 128;
            // descriptors advance by (byte offset >> 4) in their address field
            const uint64_t adesc0 = smem_desc(su32(sA), 128, sbo);
            const uint64_t bdesc0 = smem_desc(su32(sB), 128, sbo);
            TileWalk tw{ntn, R, 0, 0};
            tw.start(t0);
            int arow = -1, aloads = 0;
            for (int it = 0; it < ntiles && ok; it++, tw.next()) {
                if (tw.I != arow) {
                    if (aloads > 0) mma_commit(bar[1]);          // A may be replaced once these MMAs finish
                    ok = mbar_wait_bounded(bar[0], aloads & 1);
                    if (!ok) break;
                    arow = tw.I;
                    aloads++;
                }
                const int st = it & 1;
                ok = mbar_wait_bounded(bar[2 + st], (it >> 1) & 1);
                if (ok && it >= 1) ok = mbar_wait_bounded(bar[7], (it - 1) & 1);
                if (!ok) break;
                tc_fence_after();
                const uint64_t bst = bdesc0 + (uint64_t)((st * bstage) >> 4);
                for (int o = 0; o < NOUT; o++) {
                    for (int l = 0; l < S; l++) {
                        const uint32_t dcol = (uint32_t)((o * S + l) * TN);
                        for (int i = 0; i <= l; i++) {
                            const uint64_t ad = adesc0 + (uint64_t)((i * a_bytes) >> 4);
                            const uint64_t bd = bst + (uint64_t)(((o * kSplitMaxSlices + (l - i)) * b_bytes) >> 4);
                            for (int kc = 0; kc < kk / 32; kc++)
                                mma_i8(tmem + dcol, ad + (uint64_t)(kc * 16), bd + (uint64_t)(kc * 16), idesc,
                                       (i > 0 || kc > 0) ? 1u : 0u);
                        }
                    }
                }
                mma_commit(bar[4 + st]);     // B stage free once these MMAs are done
                mma_commit(bar[6]);          // accumulators ready
            }
            if (!ok) atomicExch(s_fail, 1);
        }
    } else {
        // ---------------- epilogue (warps 2-9), thread = tile row
        const int quarter = warp & 3;
        const int h = (warp - 2) >> 2;
        const int lane_row = quarter * 32 + lane;
        double *Wd = reinterpret_cast<double *>(W_all) + (int64_t)NOUT * b * (int64_t)n * n;
        TileWalk tw{ntn, R, 0, 0};
        tw.start(t0);
        double2 cv[NV];
        auto load_c = [&](const TileWalk &w) {
            const int arow = k1 + w.I * TM + lane_row;
            const int bc0 = k1 + w.J * TN + h * CW;
            const double2 *src = reinterpret_cast<const double2 *>(Wd + NOUT * ((int64_t)arow * n + bc0));
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const int bcol = bc0 + (2 * v) / NOUT;
                const bool any = arow < n && bcol < n && (bcol + (NOUT == 1 ? 1 : 0)) > arow;
                cv[v] = any ? src[v] : make_double2(0.0, 0.0);
            }
        };
        load_c(tw);
        for (int it = 0; it < ntiles && ok; it++) {
            ok = mbar_wait_bounded(bar[6], it & 1);
            if (!ok) break;
            tc_fence_after();
            const int arow = k1 + tw.I * TM + lane_row;
            const int bc0 = k1 + tw.J * TN + h * CW;
            const int ea = arow < n ? __ldg(&sa.ex[b * n + arow]) : 0;
            double *dst = Wd + NOUT * ((int64_t)arow * n + bc0);
            // 8 columns at a time: the S levels folded exactly into hi / lo
#pragma unroll
            for (int c8 = 0; c8 < CW / 8; c8++) {
                double dv[NOUT][8];
#pragma unroll
                for (int o = 0; o < NOUT; o++) {
                    long long hi[8], lo[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) { hi[c] = 0; lo[c] = 0; }
#pragma unroll
                    for (int l0 = 0; l0 < kSplitMaxSlices; l0 += 2) {
                        int32_t v[2][8];
#pragma unroll
                        for (int li = 0; li < 2; li++)
                            if (l0 + li < S)
                                tmem_ld8(tmem + ((uint32_t)(quarter * 32) << 16) +
                                             (uint32_t)((o * S + l0 + li) * TN + h * CW + c8 * 8), v[li]);
                        tmem_ld_wait();
#pragma unroll
                        for (int li = 0; li < 2; li++) {
                            const int l = l0 + li;
                            if (l < S) {
#pragma unroll
                                for (int c = 0; c < 8; c++) {
                                    if (l <= 3) hi[c] += (long long)v[li][c] << (7 * (3 - l));
                                    else lo[c] += (long long)v[li][c] << (7 * (6 - l));
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int c = 0; c < 8; c++) dv[o][c] = fma((double)lo[c], 0x1p-56, (double)hi[c] * 0x1p-35);
                }
                if (c8 == CW / 8 - 1) {
                    // every TMEM read of this tile is done: the MMA thread may go on
                    tc_fence_before();
                    mbar_arrive(bar[7]);
                }
                if (arow < n) {
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const int col = c8 * 8 + c, bcol = bc0 + col;
                        if (bcol < n && bcol > arow) {
                            const int e = ea + __ldg(&sa.ex[b * n + bcol]);
#pragma unroll
                            for (int o = 0; o < NOUT; o++) {
                                const int idx = NOUT * col + o;        // position in the row segment
                                const double old = (idx & 1) ? cv[idx >> 1].y : cv[idx >> 1].x;
                                dst[idx] = old + scalbn(dv[o][c], e);
                            }
                        }
                    }
                }
            }
            tw.next();
            if (it + 1 < ntiles) load_c(tw);
        }
        if (!ok) atomicExch(s_fail, 1);
    }

    tc_fence_before();
    __syncthreads();
    if (tid == 0 && *s_fail) atomicExch(&sa.err[b], PFB_ERR_TIMEOUT);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// At least 116 KB, so that a single CTA (which holds all 512 TMEM columns)
// is resident per SM and no allocation ever waits for another CTA.
template <int TN, int NOUT>
static size_t split_smem_bytes(int kk)
{
    const size_t need = (size_t)kSplitMaxSlices * kSplitTileM * kk + 2 * (size_t)NOUT * kSplitMaxSlices * TN * kk +
                        8 * 8 + 16;
    return need < 116 * 1024 ? 116 * 1024 : need;
}

template <int TN, int NOUT>
static int launch_split_t(void *W, int n, int k0, int K, int64_t batch, MatState *st, const SplitArgs &sa,
                          cudaStream_t stream)
{
    const int m = n - (k0 + K);
    const int ntn = (m + TN - 1) / TN;
    const int ntm = (m + kSplitTileM - 1) / kSplitTileM;
    int tiles = 0;
    for (int I = 0; I < ntm; I++) tiles += ntn - I * (kSplitTileM / TN) > 0 ? ntn - I * (kSplitTileM / TN) : 0;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // at most one CTA per SM over the whole batch, at least two tiles per CTA
    int per = (int)(sms / batch);
    if (per > (tiles + 1) / 2) per = (tiles + 1) / 2;
    if (per < 1) per = 1;
    auto k = split_update_kernel<TN, NOUT>;
    const size_t smem = split_smem_bytes<TN, NOUT>(sa.kk);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return PFB_ERR_CUDA;
    k<<<dim3((unsigned)per, (unsigned)batch), kSplitThreads, smem, stream>>>(W, n, k0, K, st, sa);
    return cudaGetLastError() == cudaSuccess ? PFB_OK : PFB_ERR_CUDA;
}

int launch_split_update(bool cplx, void *W, int n, int k0, int K, int64_t batch, MatState *st,
                        const SplitArgs &sa, cudaStream_t stream)
{
    if (n - (k0 + K) <= 0) return PFB_OK;
    // NOUT * S levels * TN columns <= 448 of the 512 TMEM columns
    if (!cplx) return launch_split_t<64, 1>(W, n, k0, K, batch, st, sa, stream);
    return launch_split_t<32, 2>(W, n, k0, K, batch, st, sa, stream);
}

}  // namespace pfb
