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
#include <cuda.h>
#include <limits.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "split.cuh"
#include "large.cuh"
#include "tma.cuh"

namespace pfb {

constexpr int kSplitThreads = 576;   // warp 0: loads, warp 1: MMA, warps 2-17: epilogue
constexpr int kEpiThreads = 512;

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
    a.epilogue = PFB_EPILOGUE_ROUNDTRIP;
    a.fail_b = -1;
    return a;
}

// ------------------------------------------------------------- PTX wrappers

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
// The same product with A (128 rows x 32 int8 per lane: K packed four to a
// column) in tensor memory at column address tmem_a.
PFB_D void mma_i8_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}"
                 ::"r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}
// 128 rows x 32 bytes of a K-major operand in shared memory (descriptor sdesc)
// into 128 lanes x 8 columns of tensor memory at taddr, ordered with the
// issuing thread's later MMAs.
PFB_D void tmem_cp_128x256b(uint32_t taddr, uint64_t sdesc)
{
    asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(taddr), "l"(sdesc) : "memory");
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
PFB_D void tmem_ld4(uint32_t taddr, int32_t (&v)[4])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "r"(taddr));
}
PFB_D void tmem_ld8(uint32_t taddr, int32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

// Upper-triangle tiles of the trailing block in row-major order: row tile I
// (TM rows) holds column tiles J = I*R .. ntn-1, R = TM/TN.  A CTA walks its
// range backwards (step): the first row tile, which holds the next panel's
// rows, is then among the last tiles written and still in L2 when the next
// panel kernel loads it.
struct TileWalk {
    int ntn, R, I, J;
    PFB_D void start(int idx)
    {
        I = 0;
        while (idx >= ntn - I * R) { idx -= ntn - I * R; I++; }
        J = I * R + idx;
    }
    PFB_D void step()
    {
        if (--J < I * R) { I--; J = ntn - 1; }
    }
};

// ------------------------------------------------- tensor-map (TMA) helpers

PFB_D void tma_store_3d(const CUtensorMap *map, int x, int y, int z, uint32_t src)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];"
                 ::"l"(map), "r"(x), "r"(y), "r"(z), "r"(src) : "memory");
}
PFB_D void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
PFB_D void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
PFB_D void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
PFB_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// dst[i] += src[i] for `bytes` / 8 doubles, performed by the L2 (an
// asynchronous bulk reduction from shared memory, tracked by bulk groups)
PFB_D void bulk_reduce_add_f64(double *dst, uint32_t src, uint32_t bytes)
{
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;"
                 ::"l"(dst), "r"(src), "r"(bytes) : "memory");
}
PFB_D void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
PFB_D void epi_sync() { asm volatile("bar.sync 1, 512;" ::: "memory"); }
// AND of p over the 512 epilogue threads (a barrier all of them reach), so that
// a timed-out wait ends the loop of every epilogue thread together
PFB_D bool epi_all(bool p)
{
    uint32_t r;
    asm volatile("{\n\t.reg .pred pi, po;\n\t"
                 "setp.ne.u32 pi, %1, 0;\n\t"
                 "bar.red.and.pred po, 1, 512, pi;\n\t"
                 "selp.u32 %0, 1, 0, po;\n\t}"
                 : "=r"(r) : "r"((uint32_t)p) : "memory");
    return r != 0;
}

// 2^e as a double: built from its bits in the normal range, else by scalbn
// (subnormal and overflowing powers).
PFB_D double exp2i(int e)
{
    if (e >= -1022 && e <= 1023) return __longlong_as_double((long long)(e + 1023) << 52);
    return scalbn(1.0, e);
}

// The tile scale 2^(ea + eb - 56): from its exponent bits when the warp's
// scales are all in the normal range (fast, decided by one vote), else exp2i.
PFB_D bool scales_normal(int ea, int eb, bool has_eb)
{
    const int a0 = __reduce_min_sync(0xffffffffu, ea), a1 = __reduce_max_sync(0xffffffffu, ea);
    const int b0 = __reduce_min_sync(0xffffffffu, has_eb ? eb : INT_MAX);
    const int b1 = __reduce_max_sync(0xffffffffu, has_eb ? eb : INT_MIN);
    return a0 + b0 - 56 >= -1022 && a1 + b1 - 56 <= 1023;
}
PFB_D double scale2(int ea, int eb, bool fast)
{
    return fast ? __hiloint2double((ea + eb - 56 + 1023) << 20, 0) : exp2i(ea + eb - 56);
}

// An integer |v| < 2^51 as a double, exactly, by the usual magic-number
// construction (integer add, one FP64 subtraction): it keeps the conversions
// off the transcendental/conversion pipe, which otherwise limits the epilogue.
PFB_D double i2d_exact(long long v)
{
    return __longlong_as_double(v + 0x4338000000000000LL) - 0x1.8p52;
}

// sum_l P_l 2^(7(6-l)) for the S <= 7 digit levels of one output (|P_l| < 2^23):
// adjacent levels pair up exactly in int32 (P_l * 2^7 + P_(l+1) < 2^31), the
// pairs into H = Q01 2^14 + Q23 (< 2^46) and L = Q45 2^7 + P_6 (< 2^38) in
// int64, and the value H 2^21 + L is formed with a single rounding.
PFB_D double fold_levels(const int32_t (&P)[kSplitMaxSlices])
{
    const int32_t q01 = P[0] * 128 + P[1];
    const int32_t q23 = P[2] * 128 + P[3];
    const int32_t q45 = P[4] * 128 + P[5];
    const long long hi = ((long long)q01 << 14) + q23;
    const long long lo = ((long long)q45 << 7) + P[6];
    return fma(i2d_exact(hi), 0x1p21, i2d_exact(lo));
}

// The C tile (128 rows x 64 doubles) moves as 4 boxes of 16 doubles x 128 rows
// with the 128-byte swizzle: double d of row r sits at byte
//   (d / 16) * 16384 + r * 128 + (((d % 16) / 2) ^ (r % 8)) * 16 + (d % 2) * 8,
// so the epilogue's row-per-thread 16-byte accesses are free of bank conflicts.
constexpr int kCBoxCols = 16;
constexpr int kCBoxBytes = kCBoxCols * kSplitTileM * 8;    // 16 KB
constexpr int kCTileBytes = 4 * kCBoxBytes;                // 64 KB
PFB_D uint32_t cswz(int r, int d)
{
    return (uint32_t)((d >> 4) * kCBoxBytes + r * 128 + ((((d & 15) >> 1) ^ (r & 7)) << 4));
}

// The delta tile of the reduce-add epilogue (RED): 128 rows of 64 doubles,
// row-major with a row stride of 66 doubles (528 bytes: 16-byte aligned rows,
// and the 16-byte stores of one row per lane fall on all 32 banks per quarter
// warp).
constexpr int kDeltaLd = 66;
constexpr int kDeltaTileBytes = kSplitTileM * kDeltaLd * 8;   // 67,584

// Persistent, warp-specialised update of the upper-triangle (128 x TN) tiles
// of one matrix's trailing block (blockIdx.y = matrix, blockIdx.x = CTA):
//   warp 0   bulk copies of the int8 operand chunks,
//   warp 1   one thread issues the tcgen05 MMAs,
//   warps 2-17 epilogue: warp w reads TMEM lane quarter w%4 (the only one it
//            may access) and column group h = (w-2)/4 of the tile (16 of
//            its 64 doubles, one C box); four warps per lane quarter hide
//            the latencies of the TMEM reads and the shared-memory update.
// The FP64 tile of W (C) travels by TMA in both directions: one epilogue
// thread loads the tile after next into one of two shared buffers while the
// current one is updated in place, then stores it back with a bulk tensor store
// (out-of-range rows and columns are zero-filled on load and clipped on store;
// the whole tile is written, including the part below the diagonal of diagonal
// tiles, which the factorisation never reads).  Each CTA walks a contiguous
// range of tiles, so consecutive tiles mostly share the A operand (the 128
// trailing rows), which stays in shared memory.  The S digit-level accumulators
// of a tile (NOUT * S * TN <= 448 TMEM columns) are handed back to the MMA
// thread once the epilogue has read them and, for real input, finished its
// read-modify-write: the next tile's MMAs read their operands from shared
// memory, and run alongside the read-modify-write both slowed down (a clock64
// trace at 2n = 4096: 8.4k cycles a tile that way, 7.8k in turn).  The C store,
// the next C load and the epilogue's waits still overlap the MMAs.
//
// Epilogue arithmetic: the tile value is 2^(e_a+e_b-56) * sum_l P_l 2^(7(6-l))
// (fold_levels), added to C with one fused multiply-add.
//
// RED (the reduce-add epilogue): C never comes into the SM.  The epilogue
// writes the tile's increment delta = value * 2^(e_a+e_b-56) (exact: a power
// of two times a double) into a shared-memory delta tile, and each epilogue
// warp hands eight of its rows to the L2 as bulk reduce-adds (C += delta, one
// rounding: the same result as the fused multiply-add).  The C load, the
// read-modify-write and the store leave the SM's critical path; two delta
// tiles alternate, one filled while the L2 reads the other.
//
// KK (the K of the int8 products) and S (digit slices) are template
// parameters: with them the MMA issue loop unrolls into constant descriptor
// offsets.  (A loop with run-time bounds issued one MMA per ~130 cycles on
// B200, against ~54 unrolled: the issue, not the tensor pipe, was the limit.)
template <int TN, int NOUT, int KK, int S, bool RED>
__global__ void __launch_bounds__(kSplitThreads, 1)
split_update_kernel(const __grid_constant__ CUtensorMap cmap, double *__restrict__ Wd, int n, int k0, int K,
                    MatState *__restrict__ st_all, SplitArgs sa)
{
    constexpr int TM = kSplitTileM;
    constexpr uint32_t TMEM_COLS = 512;
    constexpr int CW = TN / 4;                  // logical columns per epilogue thread
    static_assert(TN * NOUT == 64, "a C tile is 64 doubles wide");
    static_assert(NOUT * S * TN <= 448, "the S accumulators of a tile fit in TMEM");
    // The A digits of slices 0 .. kTmemA-1 live in tensor memory after the
    // accumulators (K/4 columns a slice), so their MMAs read only B from shared
    // memory: an int8 MMA of 128 x 64 x 32 reading both operands from shared
    // memory (6 KB) is bound by its bandwidth, not by the tensor pipe.
    constexpr int kAcol0 = NOUT * S * TN;
    // When the epilogue hands the accumulators back: real input (one output,
    // 64-column MMAs) after its shared-memory read-modify-write, since the next
    // tile's MMAs and that read-modify-write slow each other (update 21.6 ->
    // 20.6 ms per call at 2n = 4096); complex input (two outputs, 32-column
    // MMAs) right after reading them, where the overlap still pays (31.6
    // against 32.6 ms at 2n = 2048).
    constexpr bool kLateRelease = NOUT == 1;
    constexpr int kTmemA = (512 - kAcol0) / (KK / 4) < S ? (512 - kAcol0) / (KK / 4) : S;
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int kk = KK;
    constexpr int a_bytes = TM * kk;            // one slice of the A tile
    constexpr int b_bytes = TN * kk;            // one slice of one B tile
    unsigned char *sC = smem;                                   // 2 C tiles or 2 delta tiles, 1024-aligned
    unsigned char *sA = sC + 2 * (RED ? kDeltaTileBytes : kCTileBytes);
    unsigned char *sB = sA + kSplitMaxSlices * a_bytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + NOUT * kSplitMaxSlices * b_bytes);
    // bars: 0 a_full, 1 a_empty, 2 b_full, 3 b_empty, 4 acc_full, 5 acc_empty, 6-7 c_full
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
    // the polls of every wait of the pipeline (the drain after a failure below
    // keeps the full bound): none for the matrix PFB_SPLIT_TEST_TIMEOUT marks
    const long long lim = ((int)b == sa.fail_b) ? 0 : kWaitSpins;
    // mbarrier i sits at bar0 + 8 i (an address, not an array: a runtime index
    // into a register array would move it to local memory)
    const uint32_t bar0 = su32(bars);
    auto mb = [bar0](int i) { return bar0 + 8u * (uint32_t)i; };
    if (tid == 0) {
        for (int i = 0; i < 8; i++) mbar_init(mb(i), i == 5 ? (uint32_t)kEpiThreads : 1u);
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
    // copies in flight, for the drain on a failure: A loads issued, B loads
    // issued (producer), C loads issued and consumed (epilogue leader)
    int p_aloads = 0, p_bloads = 0, c_issued = 0, c_done = 0, m_issued = 0;

    if (warp == 0) {
        // ---------------- producer of the int8 operands
        if (lane == 0) {
            const int64_t chunk = (int64_t)TM * kk;
            TileWalk tw{ntn, R, 0, 0};
            tw.start(t1 - 1);
            int arow = -1, aloads = 0;
            for (int it = 0; it < ntiles && ok; it++, tw.step()) {
                if (tw.I != arow) {
                    if (aloads > 0) ok = mbar_wait_bounded(mb(1), (aloads - 1) & 1, lim);
                    if (!ok) break;
                    mbar_expect_tx(mb(0), (uint32_t)(S * a_bytes));
                    for (int s = 0; s < S; s++)
                        bulk_g2s(su32(sA + s * a_bytes),
                                 sa.xs + b * sa.mstride + ((int64_t)s * sa.ntile + tw.I) * chunk, a_bytes, mb(0));
                    arow = tw.I;
                    aloads++;
                    p_aloads = aloads;
                }
                if (it >= 1) ok = mbar_wait_bounded(mb(3), (it - 1) & 1, lim);
                if (!ok) break;
                const int jrow = tw.J * TN;
                const int64_t boff = (int64_t)(jrow / TM) * chunk + (int64_t)((jrow % TM) >> 3) * (kk >> 4) * 128;
                mbar_expect_tx(mb(2), (uint32_t)(S * NOUT * b_bytes));
                for (int s = 0; s < S; s++) {
                    bulk_g2s(su32(sB + s * b_bytes), sa.ys + b * sa.mstride + (int64_t)s * sa.ntile * chunk + boff,
                             b_bytes, mb(2));
                    if (NOUT == 2)
                        bulk_g2s(su32(sB + (kSplitMaxSlices + s) * b_bytes),
                                 sa.ys2 + b * sa.mstride + (int64_t)s * sa.ntile * chunk + boff, b_bytes, mb(2));
                }
                p_bloads = it + 1;
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
            tw.start(t1 - 1);
            int arow = -1, aloads = 0;
            for (int it = 0; it < ntiles && ok; it++, tw.step()) {
                if (tw.I != arow) {
                    if (aloads > 0) {
                        mma_commit(mb(1));          // A may be replaced once these MMAs finish
                        // and the tensor-memory image of A is rewritten below
                        if (kTmemA > 0) ok = mbar_wait_bounded(mb(1), (aloads - 1) & 1, lim);
                        if (!ok) break;
                    }
                    ok = mbar_wait_bounded(mb(0), aloads & 1, lim);
                    if (!ok) break;
                    tc_fence_after();
#pragma unroll
                    for (int i = 0; i < kTmemA; i++)
#pragma unroll
                        for (int kc = 0; kc < kk / 32; kc++)
                            tmem_cp_128x256b(tmem + kAcol0 + (uint32_t)(i * (kk / 4) + kc * 8),
                                             adesc0 + (uint64_t)(((i * a_bytes) >> 4) + kc * 16));
                    arow = tw.I;
                    aloads++;
                }
                ok = mbar_wait_bounded(mb(2), it & 1, lim);
                if (ok && it >= 1) ok = mbar_wait_bounded(mb(5), (it - 1) & 1, lim);
                if (!ok) break;
                tc_fence_after();
#pragma unroll
                for (int o = 0; o < NOUT; o++) {
#pragma unroll
                    for (int l = 0; l < S; l++) {
                        const uint32_t dcol = (uint32_t)((o * S + l) * TN);
#pragma unroll
                        for (int i = 0; i <= l; i++) {
                            const uint64_t ad = adesc0 + (uint64_t)((i * a_bytes) >> 4);
                            const uint64_t bd = bdesc0 + (uint64_t)(((o * kSplitMaxSlices + (l - i)) * b_bytes) >> 4);
#pragma unroll
                            for (int kc = 0; kc < kk / 32; kc++) {
                                if (i < kTmemA)
                                    mma_i8_ts(tmem + dcol, tmem + kAcol0 + (uint32_t)(i * (kk / 4) + kc * 8),
                                              bd + (uint64_t)(kc * 16), idesc, (i > 0 || kc > 0) ? 1u : 0u);
                                else
                                    mma_i8(tmem + dcol, ad + (uint64_t)(kc * 16), bd + (uint64_t)(kc * 16), idesc,
                                           (i > 0 || kc > 0) ? 1u : 0u);
                            }
                        }
                    }
                }
                mma_commit(mb(3));          // B free once these MMAs are done
                mma_commit(mb(4));          // accumulators ready
                m_issued = it + 1;
            }
            if (!ok) atomicExch(s_fail, 1);
        }
    } else if constexpr (RED) {
        // ---------------- epilogue (warps 2-17), thread = tile row; C += delta in the L2
        const int quarter = warp & 3;
        const int h = (warp - 2) >> 2;              // column group: 16 doubles
        const int r = quarter * 32 + lane;          // row within the tile
        const int e = warp - 2;                     // this warp hands rows 8e .. 8e+7 to the L2
        double *Wb = Wd + b * (int64_t)NOUT * n * n;
        TileWalk tw{ntn, R, 0, 0};
        tw.start(t1 - 1);
        for (int it = 0; it < ntiles && ok; it++) {
            const int buf = it & 1;
            const int arow = k1 + tw.I * TM + r;
            const int bc0 = k1 + tw.J * TN + h * CW;
            const int ea = arow < n ? __ldg(&sa.ex[b * n + arow]) : 0;
            const int eb_l = (lane < CW && bc0 + lane < n) ? __ldg(&sa.ex[b * n + bc0 + lane]) : 0;
            // every scale of this warp's block (its rows' ea against its
            // columns' eb) is a normal power of two
            const bool fast = scales_normal(ea, eb_l, lane < CW);
            ok = epi_all(mbar_wait_bounded(mb(4), it & 1, lim));
            if (!ok) break;
            tc_fence_after();
            double dv[NOUT][CW];
#pragma unroll
            for (int c8 = 0; c8 < CW / 8; c8++) {
#pragma unroll
                for (int o = 0; o < NOUT; o++) {
                    int32_t v[S][8];
#pragma unroll
                    for (int l = 0; l < S; l++)
                        tmem_ld8(tmem + ((uint32_t)(quarter * 32) << 16) +
                                     (uint32_t)((o * S + l) * TN + h * CW + c8 * 8), v[l]);
                    tmem_ld_wait();
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        int32_t P[kSplitMaxSlices];
#pragma unroll
                        for (int l = 0; l < kSplitMaxSlices; l++) P[l] = l < S ? v[l < S ? l : 0][c] : 0;
                        dv[o][c8 * 8 + c] = fold_levels(P);
                    }
                }
            }
            if constexpr (!kLateRelease) {
                tc_fence_before();
                mbar_arrive(mb(5));
            }
            // this delta tile was last read by the reduce-adds of tile it - 2
            if (lane == 0 && it >= 2) bulk_wait_read1();
            epi_sync();
            double *db = reinterpret_cast<double *>(sC + buf * kDeltaTileBytes);
#pragma unroll
            for (int c8 = 0; c8 < CW / 8; c8++) {
                double sc[8];
#pragma unroll
                for (int c = 0; c < 8; c++) sc[c] = scale2(ea, __shfl_sync(0xffffffffu, eb_l, c8 * 8 + c), fast);
                const int d0 = h * 16 + c8 * 8 * NOUT;
#pragma unroll
                for (int pr = 0; pr < 4 * NOUT; pr++) {
                    double2 v;
                    if (NOUT == 1) {
                        v.x = dv[0][c8 * 8 + 2 * pr] * sc[2 * pr];
                        v.y = dv[0][c8 * 8 + 2 * pr + 1] * sc[2 * pr + 1];
                    } else {
                        v.x = dv[0][c8 * 8 + pr] * sc[pr];
                        v.y = dv[NOUT - 1][c8 * 8 + pr] * sc[pr];
                    }
                    *reinterpret_cast<double2 *>(db + r * kDeltaLd + d0 + 2 * pr) = v;
                }
            }
            if constexpr (kLateRelease) {   // as in the round trip
                tc_fence_before();
                mbar_arrive(mb(5));
            }
            fence_proxy_async();
            epi_sync();
            if (lane == 0) {
                const int c0 = k1 + tw.J * TN;
                const int cols = (n - c0 < TN) ? n - c0 : TN;      // even: n and c0 are
                const uint32_t bytes = (uint32_t)(cols * NOUT * 8);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int rr = 8 * e + i;
                    const int a = k1 + tw.I * TM + rr;
                    if (a < n)
                        bulk_reduce_add_f64(Wb + (int64_t)a * NOUT * n + (int64_t)NOUT * c0,
                                            su32(db + rr * kDeltaLd), bytes);
                }
                bulk_commit();
            }
            tw.step();
        }
        // every reduce-add has landed before the CTA exits
        if (lane == 0) bulk_wait0();
        if (!ok) atomicExch(s_fail, 1);
    } else {
        // ---------------- epilogue (warps 2-17), thread = tile row
        const bool leader = tid == 64;
        const int quarter = warp & 3;
        const int h = (warp - 2) >> 2;              // column group: 16 doubles = one C box
        const int r = quarter * 32 + lane;          // row within the tile
        const int bz = (int)b;
        TileWalk tw{ntn, R, 0, 0};
        tw.start(t1 - 1);
        TileWalk tl = tw;                           // the leader's load cursor, one tile ahead
        // (tile coordinates are passed by value: a reference would put the
        // cursors in local memory)
#define PFB_LOAD_C(buf, I_, J_)                                                                          \
    do {                                                                                                \
        c_issued++;                                                                                     \
        mbar_expect_tx(mb(6 + (buf)), (uint32_t)kCTileBytes);                                          \
        const int y_ = k1 + (I_) * TM, x0_ = NOUT * (k1 + (J_) * TN);                                   \
        _Pragma("unroll") for (int q = 0; q < 4; q++)                                                   \
            tma_load_3d(su32(sC + (buf) * kCTileBytes + q * kCBoxBytes), &cmap, x0_ + q * kCBoxCols, y_, bz, \
                        mb(6 + (buf)));                                                                \
    } while (0)
        if (leader) {
            PFB_LOAD_C(0, tl.I, tl.J);
            tl.step();
            if (ntiles > 1) PFB_LOAD_C(1, tl.I, tl.J);
        }
        for (int it = 0; it < ntiles && ok; it++) {
            const int buf = it & 1;
            // this tile's scale exponents, loaded before the waits: the row's
            // own, and lane c's the one of column c of this thread's group
            const int arow = k1 + tw.I * TM + r;
            const int bc0 = k1 + tw.J * TN + h * CW;
            const int ea = arow < n ? __ldg(&sa.ex[b * n + arow]) : 0;
            const int eb_l = (lane < CW && bc0 + lane < n) ? __ldg(&sa.ex[b * n + bc0 + lane]) : 0;
            // every scale of this warp's block (its rows' ea against its
            // columns' eb) is a normal power of two
            const bool fast = scales_normal(ea, eb_l, lane < CW);
            bool w_ok = mbar_wait_bounded(mb(6 + buf), (it >> 1) & 1, lim);
            if (w_ok) c_done = it + 1;
            if (w_ok) w_ok = mbar_wait_bounded(mb(4), it & 1, lim);
            ok = epi_all(w_ok);
            if (!ok) break;
            if (kLateRelease && leader && it >= 1 && it + 1 < ntiles) {
                // load tile it+1 into the buffer of tile it-1 (whose store,
                // issued a phase ago, has read it by now) before the fold: its
                // shared-memory writes then overlap the fold's TMEM reads and
                // integer work instead of the read-modify-write below
                bulk_wait_read0();
                tl.step();
                PFB_LOAD_C(buf ^ 1, tl.I, tl.J);
            }
            tc_fence_after();
            unsigned char *cb = sC + buf * kCTileBytes;
            // all of this thread's TMEM values first, folded to one double per
            // output (CW * NOUT registers)
            double dv[NOUT][CW];
#pragma unroll
            for (int c8 = 0; c8 < CW / 8; c8++) {
#pragma unroll
                for (int o = 0; o < NOUT; o++) {
                    int32_t v[S][8];
#pragma unroll
                    for (int l = 0; l < S; l++)
                        tmem_ld8(tmem + ((uint32_t)(quarter * 32) << 16) +
                                     (uint32_t)((o * S + l) * TN + h * CW + c8 * 8), v[l]);
                    tmem_ld_wait();
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        int32_t P[kSplitMaxSlices];
#pragma unroll
                        for (int l = 0; l < kSplitMaxSlices; l++) P[l] = l < S ? v[l < S ? l : 0][c] : 0;
                        dv[o][c8 * 8 + c] = fold_levels(P);
                    }
                }
            }
            if constexpr (!kLateRelease) {
                tc_fence_before();
                mbar_arrive(mb(5));
                if (leader && it >= 1 && it + 1 < ntiles) {
                    // complex input: the next C tile is loaded here, after the
                    // fold, where it was measured
                    bulk_wait_read0();
                    tl.step();
                    PFB_LOAD_C(buf ^ 1, tl.I, tl.J);
                }
            }
            // read-modify-write of the CW * NOUT doubles in shared memory:
            // C += value * 2^(ea + eb - 56), one rounding.  A chunk's loads are
            // all issued before its stores, so their latencies overlap.
#pragma unroll
            for (int c8 = 0; c8 < CW / 8; c8++) {
                double sc[8];
#pragma unroll
                for (int c = 0; c < 8; c++) sc[c] = scale2(ea, __shfl_sync(0xffffffffu, eb_l, c8 * 8 + c), fast);
                const int d0 = h * 16 + c8 * 8 * NOUT;
                double2 old[4 * NOUT];
#pragma unroll
                for (int pr = 0; pr < 4 * NOUT; pr++) old[pr] = *reinterpret_cast<const double2 *>(cb + cswz(r, d0 + 2 * pr));
#pragma unroll
                for (int pr = 0; pr < 4 * NOUT; pr++) {
                    if (NOUT == 1) {
                        old[pr].x = fma(dv[0][c8 * 8 + 2 * pr], sc[2 * pr], old[pr].x);
                        old[pr].y = fma(dv[0][c8 * 8 + 2 * pr + 1], sc[2 * pr + 1], old[pr].y);
                    } else {
                        old[pr].x = fma(dv[0][c8 * 8 + pr], sc[pr], old[pr].x);
                        old[pr].y = fma(dv[NOUT - 1][c8 * 8 + pr], sc[pr], old[pr].y);
                    }
                }
#pragma unroll
                for (int pr = 0; pr < 4 * NOUT; pr++) *reinterpret_cast<double2 *>(cb + cswz(r, d0 + 2 * pr)) = old[pr];
            }
            // real input: the accumulators go back to the MMA thread only now
            // (kLateRelease)
            if constexpr (kLateRelease) {
                tc_fence_before();
                mbar_arrive(mb(5));
            }
            // the tile in shared memory is complete: one thread stores it
            fence_proxy_async();
            epi_sync();
            if (leader) {
                const int y = k1 + tw.I * TM, x0 = NOUT * (k1 + tw.J * TN);
#pragma unroll
                for (int q = 0; q < 4; q++)
                    tma_store_3d(&cmap, x0 + q * kCBoxCols, y, bz, su32(cb + q * kCBoxBytes));
                bulk_commit();
            }
            tw.step();
        }
#undef PFB_LOAD_C
        if (leader) bulk_wait0();
        if (!ok) atomicExch(s_fail, 1);
    }

    tc_fence_before();
    __syncthreads();
    if (*s_fail) {
        // a wait gave up: let this CTA's copies in flight land (bounded) before exit
        if (tid == 0) {
            if (p_aloads > 0) mbar_wait_bounded(mb(0), (p_aloads - 1) & 1);
            if (p_bloads > 0) mbar_wait_bounded(mb(2), (p_bloads - 1) & 1);
            atomicExch(&sa.err[b], PFB_ERR_TIMEOUT);
        }
        if (tid == 32 && m_issued > 0) mbar_wait_bounded(mb(4), (m_issued - 1) & 1);   // MMAs done
        if (tid == 64)
            for (int t = c_done; t < c_issued; t++) mbar_wait_bounded(mb(6 + (t & 1)), (t >> 1) & 1);
        __syncthreads();
    }
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ------------------------------------------- transposed tiles, direct C access

// Tiles of the transposed product for the direct epilogue: b-tile I covers 128
// trailing columns (the MMA's M, TMEM lanes), a-tile J covers TN trailing rows
// (the MMA's N, TMEM columns; R = 128 / TN a-tiles per b-tile width); b-tile I
// meets the upper triangle in a-tiles 0 .. (I+1) R - 1.  Walked backwards from
// the end of a CTA's range, like TileWalk.
struct DirectWalk {
    int nta, R, I, J;
    PFB_D int count(int i) const { return (i + 1) * R < nta ? (i + 1) * R : nta; }
    PFB_D void start(int idx)
    {
        I = 0;
        while (idx >= count(I)) { idx -= count(I); I++; }
        J = idx;
    }
    PFB_D void step()
    {
        if (--J < 0) { I--; J = count(I) - 1; }
    }
};

// The split update with the tile transposed and the working matrix read and
// written directly from global memory (PFB_EPILOGUE_DIRECT).
//
// The MMA's A operand is the Y digits of 128 trailing columns b and its B
// operand the X digits of TN trailing rows a, so TMEM lane = column b and TMEM
// column = row a: P_l[b][a] = sum_{i+j=l} Y_j[b] . X_i[a], the same integer
// sums as split_update_kernel's (the products commute), hence the same bits.
// Complex input (NOUT = 2, TN = 32 complex rows) multiplies two A images --
// [Yr | -Yi] for the real part and [Yi | Yr] for the imaginary part -- by one B
// image [Xr | Xi].  An epilogue thread owns one column b and TN / 4
// consecutive rows a, and the 32 lanes of a warp own 32 adjacent columns:
// every load and store of C is a coalesced row segment (256 bytes real, 512
// complex).  The thread issues its loads of C before it waits for the
// accumulators (their latency hides behind the MMAs), reads the S levels from
// TMEM four rows at a time, folds them and adds them with one fused
// multiply-add per value, and stores only the strictly upper part (a < b), the
// only part the factorisation reads.  Shared memory holds operands only: the A
// image(s) of a b-tile (reused along it) and two B images, so the next tile's
// B arrives while the current one multiplies.
template <int NOUT, int KK, int S>
__global__ void __launch_bounds__(kSplitThreads, 1)   // 96 registers: 5 of the 18 warps share an SM partition
split_update_direct_kernel(double *__restrict__ W_all, int n, int k0, int K, MatState *__restrict__ st_all,
                           SplitArgs sa)
{
    constexpr int TM = kSplitTileM;             // b columns per tile (MMA M)
    constexpr int TN = 64 / NOUT;               // a rows per tile (MMA N)
    constexpr int RW = TN / 4;                  // rows per epilogue thread
    constexpr uint32_t TMEM_COLS = 512;
    static_assert(NOUT * S * TN <= 448, "the S accumulators of a tile fit in TMEM");
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int a_bytes = TM * KK;            // one slice of one A image (Y digits)
    constexpr int b_bytes = TN * KK;            // one slice of one B image (X digits)
    unsigned char *sA = smem;                                              // NOUT images
    unsigned char *sB = sA + NOUT * kSplitMaxSlices * a_bytes;             // two buffers
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + 2 * kSplitMaxSlices * b_bytes);
    // bars: 0 a_full, 1 a_empty, 2-3 b_full, 4-5 b_empty, 6 acc_full, 7 acc_empty
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 8);
    int *s_fail = reinterpret_cast<int *>(tmem_slot + 1);

    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    const int k1 = k0 + K;
    const int m = n - k1;
    const int ntb = (m + TM - 1) / TM;
    const int nta = (m + TN - 1) / TN;
    constexpr int R = TM / TN;
    DirectWalk cw{nta, R, 0, 0};
    int total = 0;
    for (int I = 0; I < ntb; I++) total += cw.count(I);
    const int t0 = (int)((int64_t)total * blockIdx.x / gridDim.x);
    const int t1 = (int)((int64_t)total * (blockIdx.x + 1) / gridDim.x);
    if (t0 >= t1) return;
    const int ntiles = t1 - t0;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long lim = ((int)b == sa.fail_b) ? 0 : kWaitSpins;
    const uint32_t bar0 = su32(bars);
    auto mb = [bar0](int i) { return bar0 + 8u * (uint32_t)i; };
    if (tid == 0) {
        for (int i = 0; i < 8; i++) mbar_init(mb(i), i == 7 ? (uint32_t)kEpiThreads : 1u);
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
    int p_aloads = 0, p_bloads = 0, m_issued = 0;
    const int64_t chunk = (int64_t)TM * KK;

    if (warp == 0) {
        // ---------------- producer of the int8 operands
        if (lane == 0) {
            DirectWalk w{nta, R, 0, 0};
            w.start(t1 - 1);
            int brow = -1, aloads = 0;
            for (int it = 0; it < ntiles && ok; it++, w.step()) {
                if (w.I != brow) {
                    if (aloads > 0) ok = mbar_wait_bounded(mb(1), (aloads - 1) & 1, lim);
                    if (!ok) break;
                    mbar_expect_tx(mb(0), (uint32_t)(NOUT * S * a_bytes));
                    for (int o = 0; o < NOUT; o++)
                        for (int q = 0; q < S; q++)
                            bulk_g2s(su32(sA + (o * kSplitMaxSlices + q) * a_bytes),
                                     (o == 0 ? sa.ys : sa.ys2) + b * sa.mstride +
                                         ((int64_t)q * sa.ntile + w.I) * chunk,
                                     a_bytes, mb(0));
                    brow = w.I;
                    aloads++;
                    p_aloads = aloads;
                }
                const int bb = it & 1;
                if (it >= 2) ok = mbar_wait_bounded(mb(4 + bb), ((it - 2) >> 1) & 1, lim);
                if (!ok) break;
                const int arow = w.J * TN;
                const int64_t boff = (int64_t)(arow / TM) * chunk + (int64_t)((arow % TM) >> 3) * (KK >> 4) * 128;
                mbar_expect_tx(mb(2 + bb), (uint32_t)(S * b_bytes));
                for (int q = 0; q < S; q++)
                    bulk_g2s(su32(sB + (bb * kSplitMaxSlices + q) * b_bytes),
                             sa.xs + b * sa.mstride + (int64_t)q * sa.ntile * chunk + boff, b_bytes, mb(2 + bb));
                p_bloads = it + 1;
            }
            if (!ok) atomicExch(s_fail, 1);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_i8(TM, TN);
            const uint32_t sbo = (uint32_t)(KK >> 4) * 128;
            const uint64_t adesc0 = smem_desc(su32(sA), 128, sbo);
            DirectWalk w{nta, R, 0, 0};
            w.start(t1 - 1);
            int brow = -1, aloads = 0;
            for (int it = 0; it < ntiles && ok; it++, w.step()) {
                if (w.I != brow) {
                    if (aloads > 0) mma_commit(mb(1));
                    ok = mbar_wait_bounded(mb(0), aloads & 1, lim);
                    if (!ok) break;
                    brow = w.I;
                    aloads++;
                }
                const int bb = it & 1;
                ok = mbar_wait_bounded(mb(2 + bb), (it >> 1) & 1, lim);
                if (ok && it >= 1) ok = mbar_wait_bounded(mb(7), (it - 1) & 1, lim);
                if (!ok) break;
                tc_fence_after();
                const uint64_t bdesc0 = smem_desc(su32(sB + bb * kSplitMaxSlices * b_bytes), 128, sbo);
#pragma unroll
                for (int o = 0; o < NOUT; o++) {
#pragma unroll
                    for (int l = 0; l < S; l++) {
                        const uint32_t dcol = (uint32_t)((o * S + l) * TN);
#pragma unroll
                        for (int i = 0; i <= l; i++) {
                            // Y digit i of the columns with X digit l - i of the rows
                            const uint64_t ad = adesc0 + (uint64_t)(((o * kSplitMaxSlices + i) * a_bytes) >> 4);
                            const uint64_t bd = bdesc0 + (uint64_t)(((l - i) * b_bytes) >> 4);
#pragma unroll
                            for (int kc = 0; kc < KK / 32; kc++)
                                mma_i8(tmem + dcol, ad + (uint64_t)(kc * 16), bd + (uint64_t)(kc * 16), idesc,
                                       (i > 0 || kc > 0) ? 1u : 0u);
                        }
                    }
                }
                mma_commit(mb(4 + bb));     // this B buffer is free once these MMAs are done
                mma_commit(mb(6));          // accumulators ready
                m_issued = it + 1;
            }
            if (!ok) atomicExch(s_fail, 1);
        }
    } else {
        // ---------------- epilogue (warps 2-17): lane = column b, RW rows a
        const int quarter = warp & 3;
        const int h = (warp - 2) >> 2;              // rows RW h .. RW h + RW - 1 of the a-tile
        double *W = W_all + b * (int64_t)NOUT * n * n;
        DirectWalk w{nta, R, 0, 0};
        w.start(t1 - 1);
        for (int it = 0; it < ntiles && ok; it++, w.step()) {
            const int col = k1 + w.I * TM + quarter * 32 + lane;     // this thread's column b
            const int row0 = k1 + w.J * TN + RW * h;                  // its first row a
            const int eb = col < n ? __ldg(&sa.ex[b * n + col]) : 0;
            const int ea_l = (lane < RW && row0 + lane < n) ? __ldg(&sa.ex[b * n + row0 + lane]) : 0;
            // C of this thread's rows, loaded before the accumulators are waited for
            double cv[RW][NOUT];
#pragma unroll
            for (int c = 0; c < RW; c++) {
                const int a = row0 + c;
                const bool up = a < col && col < n;
                const int64_t e = ((int64_t)a * n + col) * NOUT;
                if constexpr (NOUT == 1) {
                    cv[c][0] = up ? W[e] : 0.0;
                } else {
                    const double2 z = up ? *reinterpret_cast<const double2 *>(W + e) : make_double2(0.0, 0.0);
                    cv[c][0] = z.x;
                    cv[c][NOUT - 1] = z.y;
                }
            }
            ok = epi_all(mbar_wait_bounded(mb(6), it & 1, lim));
            if (!ok) break;
            tc_fence_after();
            // four rows at a time: S x 4 accumulator words per output beside C
#pragma unroll
            for (int c4 = 0; c4 < RW / 4; c4++) {
#pragma unroll
                for (int o = 0; o < NOUT; o++) {
                    int32_t v[S][4];
#pragma unroll
                    for (int l = 0; l < S; l++)
                        tmem_ld4(tmem + ((uint32_t)(quarter * 32) << 16) +
                                     (uint32_t)((o * S + l) * TN + RW * h + c4 * 4), v[l]);
                    tmem_ld_wait();
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        int32_t P[kSplitMaxSlices];
#pragma unroll
                        for (int l = 0; l < kSplitMaxSlices; l++) P[l] = l < S ? v[l < S ? l : 0][c] : 0;
                        const double sc = exp2i(eb + __shfl_sync(0xffffffffu, ea_l, c4 * 4 + c) - 56);
                        cv[c4 * 4 + c][o] = fma(fold_levels(P), sc, cv[c4 * 4 + c][o]);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(mb(7));
#pragma unroll
            for (int c = 0; c < RW; c++) {
                const int a = row0 + c;
                if (a < col && col < n) {
                    const int64_t e = ((int64_t)a * n + col) * NOUT;
                    if constexpr (NOUT == 1) W[e] = cv[c][0];
                    else *reinterpret_cast<double2 *>(W + e) = make_double2(cv[c][0], cv[c][NOUT - 1]);
                }
            }
        }
        if (!ok) atomicExch(s_fail, 1);
    }

    tc_fence_before();
    __syncthreads();
    if (*s_fail) {
        // a wait gave up: let this CTA's copies and MMAs in flight land (bounded) before exit
        if (tid == 0) {
            if (p_aloads > 0) mbar_wait_bounded(mb(0), (p_aloads - 1) & 1);
            for (int t = (p_bloads > 2 ? p_bloads - 2 : 0); t < p_bloads; t++)
                mbar_wait_bounded(mb(2 + (t & 1)), (t >> 1) & 1);
            atomicExch(&sa.err[b], PFB_ERR_TIMEOUT);
        }
        if (tid == 32 && m_issued > 0) mbar_wait_bounded(mb(6), (m_issued - 1) & 1);
        __syncthreads();
    }
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

template <int NOUT, int KK>
static size_t split_direct_smem_bytes()
{
    return (size_t)NOUT * kSplitMaxSlices * kSplitTileM * KK + (size_t)2 * kSplitMaxSlices * (64 / NOUT) * KK +
           8 * 8 + 16;
}

template <int TN, int NOUT, bool RED>
static size_t split_smem_bytes(int kk)
{
    return (size_t)2 * (RED ? kDeltaTileBytes : kCTileBytes) + (size_t)kSplitMaxSlices * kSplitTileM * kk +
           (size_t)NOUT * kSplitMaxSlices * TN * kk + 8 * 8 + 16;
}

// W of a batch as a 3-D FP64 tensor {NOUT*n columns, n rows, batch}, boxes of
// 16 doubles x 128 rows with the 128-byte swizzle.
static bool make_c_map(CUtensorMap *map, void *W, int n, int nout, int64_t batch)
{
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nout * n, (cuuint64_t)n, (cuuint64_t)batch};
    const cuuint64_t strides[2] = {(cuuint64_t)nout * n * 8, (cuuint64_t)nout * n * n * 8};
    const cuuint32_t box[3] = {(cuuint32_t)kCBoxCols, (cuuint32_t)kSplitTileM, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, W, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int TN, int NOUT, int KK, int S, bool RED>
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
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    if (!RED && !make_c_map(&map, W, n, NOUT, batch)) return PFB_ERR_UNSUPPORTED;
    auto k = split_update_kernel<TN, NOUT, KK, S, RED>;
    const size_t smem = split_smem_bytes<TN, NOUT, RED>(KK);
    if (cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != PFB_OK) return PFB_ERR_CUDA;
    k<<<dim3((unsigned)per, (unsigned)batch), kSplitThreads, smem, stream>>>(map, static_cast<double *>(W), n,
                                                                            k0, K, st, sa);
    return launch_status();
}

template <int NOUT, int KK, int S>
static int launch_split_direct(void *W, int n, int k0, int K, int64_t batch, MatState *st, const SplitArgs &sa,
                               cudaStream_t stream)
{
    constexpr int TN = 64 / NOUT, R = kSplitTileM / TN;
    const int m = n - (k0 + K);
    const int ntb = (m + kSplitTileM - 1) / kSplitTileM;
    const int nta = (m + TN - 1) / TN;
    int tiles = 0;
    for (int I = 0; I < ntb; I++) tiles += (I + 1) * R < nta ? (I + 1) * R : nta;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per = (int)(sms / batch);
    if (per > (tiles + 1) / 2) per = (tiles + 1) / 2;
    if (per < 1) per = 1;
    auto k = split_update_direct_kernel<NOUT, KK, S>;
    const size_t smem = split_direct_smem_bytes<NOUT, KK>();
    if (cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != PFB_OK) return PFB_ERR_CUDA;
    k<<<dim3((unsigned)per, (unsigned)batch), kSplitThreads, smem, stream>>>(static_cast<double *>(W), n, k0, K, st,
                                                                            sa);
    return launch_status();
}

// one instantiation per (operand width, slices, epilogue): the MMA issue
// unrolls; the reduce-add epilogue is built for 5 to 7 digits (the counts the
// accuracy bar admits), fewer digits use the shared-memory round trip
template <int TN, int NOUT, int KK>
static int launch_split_s(void *W, int n, int k0, int K, int64_t batch, MatState *st, const SplitArgs &sa,
                          cudaStream_t stream)
{
    const bool red = sa.epilogue == PFB_EPILOGUE_REDUCE;
    if (sa.epilogue == PFB_EPILOGUE_DIRECT) {
        switch (sa.slices) {
        case 5: return launch_split_direct<NOUT, KK, 5>(W, n, k0, K, batch, st, sa, stream);
        case 6: return launch_split_direct<NOUT, KK, 6>(W, n, k0, K, batch, st, sa, stream);
        case 7: return launch_split_direct<NOUT, KK, 7>(W, n, k0, K, batch, st, sa, stream);
        default: break;   // fewer digits: the round trip below
        }
    }
    switch (sa.slices) {
    case 1: return launch_split_t<TN, NOUT, KK, 1, false>(W, n, k0, K, batch, st, sa, stream);
    case 2: return launch_split_t<TN, NOUT, KK, 2, false>(W, n, k0, K, batch, st, sa, stream);
    case 3: return launch_split_t<TN, NOUT, KK, 3, false>(W, n, k0, K, batch, st, sa, stream);
    case 4: return launch_split_t<TN, NOUT, KK, 4, false>(W, n, k0, K, batch, st, sa, stream);
    case 5:
        return red ? launch_split_t<TN, NOUT, KK, 5, true>(W, n, k0, K, batch, st, sa, stream)
                   : launch_split_t<TN, NOUT, KK, 5, false>(W, n, k0, K, batch, st, sa, stream);
    case 6:
        return red ? launch_split_t<TN, NOUT, KK, 6, true>(W, n, k0, K, batch, st, sa, stream)
                   : launch_split_t<TN, NOUT, KK, 6, false>(W, n, k0, K, batch, st, sa, stream);
    case 7:
        return red ? launch_split_t<TN, NOUT, KK, 7, true>(W, n, k0, K, batch, st, sa, stream)
                   : launch_split_t<TN, NOUT, KK, 7, false>(W, n, k0, K, batch, st, sa, stream);
    default: return PFB_ERR_INVALID;
    }
}

int launch_split_update(bool cplx, void *W, int n, int k0, int K, int64_t batch, MatState *st,
                        const SplitArgs &sa, cudaStream_t stream)
{
    if (n - (k0 + K) <= 0) return PFB_OK;
    // NOUT * S levels * TN columns <= 448 of the 512 TMEM columns
    if (cplx) {
        if (sa.kk != 64) return PFB_ERR_INVALID;
        return launch_split_s<32, 2, 64>(W, n, k0, K, batch, st, sa, stream);
    }
    if (sa.kk == 64) return launch_split_s<64, 1, 64>(W, n, k0, K, batch, st, sa, stream);
    if (sa.kk == 32) return launch_split_s<64, 1, 32>(W, n, k0, K, batch, st, sa, stream);
    return PFB_ERR_INVALID;
}

}  // namespace pfb
