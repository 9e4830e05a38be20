// ragged.cu -- (log|Pf|, sign) of a ragged batch (matrices of different even
// orders and of float32 or float64) in one persistent launch.
//
// The reference has no ragged entry point: a caller loops over sizes and calls
// slog_pfaffian (pfcuda/cuda_api.py:57-76) once per matrix or per equal-size
// group, and each call runs the host-driven loop of
// src/slog_pfaffian_lg.cu:151-211.  Here one kernel covers the whole batch:
//   * ragged_order_kernel sorts the matrix indices by order, largest first (a
//     counting sort over n/2, one CTA), so the longest factorisations start
//     first and the tail of the persistent loop is made of small ones;
//   * ragged_kernel: persistent CTAs take the next matrix from a device work
//     counter and factor it alone: copy into a private FP64 working matrix,
//     then for each NB-row panel the panel factorisation of large.cu run by a
//     single CTA (panel_body with a cluster of one) followed by an in-CTA skew
//     rank-NB update of the upper trailing block on the FP64 tensor cores.
//     A pivot step is a chain of dependent latencies (reductions, barriers,
//     the load of the interchanged row), not a throughput limit, so the
//     kernel runs two CTAs per SM, each on its own matrix, with 16-row panels
//     (the register window of 16 rows x 512 columns leaves room for two CTAs);
//     a batch holding an order above 528 runs one CTA per SM with 32-row
//     panels, whose window covers orders up to 544.
// Nothing in the call synchronises the host or allocates, so a caller can
// capture it in a CUDA graph and replay it.
#include "common.cuh"
#include "large.cuh"
#include "panel.cuh"
#include "dmma.cuh"

namespace pfb {

constexpr int kRaggedCPT = 2;        // trailing columns per thread (2 x 256 threads)
constexpr int kRaggedMaxCTAs = 320;  // workspace is sized for this many CTAs
// staged row stride of the panel rows (4 mod 16 doubles)
template <int NB> __host__ __device__ constexpr int strip_ld() { return PFB_RAGGED_MAX_N - NB + 4; }
// the two configurations: panel width, CTAs per SM, a warp's output block in the update
template <int NB> struct RaggedCfg;
template <> struct RaggedCfg<16> { static constexpr int kMinBlocks = 2, kUpdBlock = 16, kMaxN = 16 + 512; };
template <> struct RaggedCfg<32> { static constexpr int kMinBlocks = 1, kUpdBlock = 32, kMaxN = 32 + 512; };
static_assert(RaggedCfg<32>::kMaxN == PFB_RAGGED_MAX_N, "the wide configuration covers every order");

struct RaggedLayout {
    size_t order_off, counter_off, cta_off, cta_bytes, w_off, st_off, piv_off, total;
};

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

static RaggedLayout ragged_layout(int64_t count, int max_n)
{
    RaggedLayout L{};
    size_t off = 0;
    L.order_off = off;
    off = al256(off + (size_t)count * sizeof(int32_t));
    L.counter_off = off;
    off = al256(off + 256);
    L.cta_off = off;
    L.w_off = 0;
    L.st_off = al256((size_t)max_n * max_n * sizeof(double));
    L.piv_off = al256(L.st_off + sizeof(MatState));
    L.cta_bytes = al256(L.piv_off + (size_t)(max_n / 2 + 1) * sizeof(int32_t));
    L.total = off + (size_t)kRaggedMaxCTAs * L.cta_bytes;
    return L;
}

size_t ragged_workspace_bytes(int64_t count, int max_n)
{
    if (count < 0 || max_n < 0 || max_n > PFB_RAGGED_MAX_N) return 0;
    return ragged_layout(count, max_n).total;
}

// Counting sort of the matrix indices by order, largest first (one CTA).
__global__ void __launch_bounds__(1024)
ragged_order_kernel(const int32_t *__restrict__ ns, int64_t count, int32_t *__restrict__ order,
                    int *__restrict__ counter)
{
    constexpr int NBK = PFB_RAGGED_MAX_N / 2 + 2;
    __shared__ int hist[NBK];
    __shared__ int start[NBK];
    for (int i = threadIdx.x; i < NBK; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    auto bucket = [&](int64_t i) {
        const int n = ns[i];
        // larger orders first; invalid orders (rejected later) go last
        return (n < 0 || n > PFB_RAGGED_MAX_N) ? NBK - 1 : (PFB_RAGGED_MAX_N / 2 - n / 2);
    };
    for (int64_t i = threadIdx.x; i < count; i += blockDim.x) atomicAdd(&hist[bucket(i)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < NBK; k++) { start[k] = acc; acc += hist[k]; }
        *counter = 0;
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < count; i += blockDim.x) {
        const int pos = atomicAdd(&start[bucket(i)], 1);
        order[pos] = (int32_t)i;
    }
}

// In-CTA update of the upper trailing block after the panel at k0 on the FP64
// tensor cores: S22[a][b] += sum_r X[r][a] Y[r][b], X = panel rows, Y[2s] =
// X[2s+1], Y[2s+1] = -X[2s] (dmma.cuh).  The K panel rows (columns k1..n) are
// staged once in shared memory; then each warp walks its own S x S output
// blocks of the upper triangle, the next block's C loads in flight while the
// current block's m8n8k4 products run.
template <int NB, int S>
__device__ __noinline__ void cta_update(double *__restrict__ W, int n, int k0, int K,
                                        double (*P)[strip_ld<NB>()])
{
    const int k1 = k0 + K;
    const int m = n - k1;
    if (m <= 0) return;
    constexpr int F = S / 8;             // fragments per block side
    const int mp = (m + S - 1) / S * S;  // staged width; zero beyond n
    const int half = mp / 2;             // 16-byte chunks per staged row
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int e = tid; e < NB * half; e += kTT) {
        const int r = e / half, c = 2 * (e - r * half);
        const bool ok = r < K && k1 + c < n;
        cp_async16(&P[r][c], ok ? W + (int64_t)(k0 + r) * n + k1 + c : W, ok);
    }
    cp_async_commit();
    const int nb = mp / S;
    const int items = nb * (nb + 1) / 2;
    int it = warp, I = 0, J = 0;
    double acc[F][F][2], nxt[F][F][2];
    if (it < items) {
        upper_block(it, nb, I, J);
        load_c_frags<F, F>(acc, W, n, k1 + S * I, k1 + S * J);
    }
    cp_async_wait<0>();
    __syncthreads();
    while (it < items) {
        const int nx = it + kTT / 32;
        int In = 0, Jn = 0;
        if (nx < items) {
            upper_block(nx, nb, In, Jn);
            load_c_frags<F, F>(nxt, W, n, k1 + S * In, k1 + S * Jn);
        }
#pragma unroll 1
        for (int kb = 0; kb < NB; kb += 4) dmma_kstep<F, F>(acc, &P[kb][S * I], &P[kb][S * J], strip_ld<NB>());
        store_c_frags<F, F>(acc, W, n, k1 + S * I, k1 + S * J);
#pragma unroll
        for (int i = 0; i < F; i++)
#pragma unroll
            for (int j = 0; j < F; j++) {
                acc[i][j][0] = nxt[i][j][0];
                acc[i][j][1] = nxt[i][j][1];
            }
        I = In;
        J = Jn;
        it = nx;
    }
}

// W <- the matrix at A widened to FP64 (nn = n^2 elements, n even).  16-byte
// loads, eight in flight per thread, when A is 16-byte aligned; element loads
// otherwise.
__device__ __noinline__ void copy_in_item(double *__restrict__ W, const void *A, int dt, int64_t nn)
{
    constexpr int U = 8;
    const int tid = threadIdx.x;
    double2 *w2 = reinterpret_cast<double2 *>(W);
    if (((uintptr_t)A & 15) == 0 && dt == PFB_F64) {
        const double2 *a = static_cast<const double2 *>(A);
        const int64_t m = nn / 2;
        for (int64_t e = tid; e < m; e += U * kTT) {
            double2 v[U];
#pragma unroll
            for (int u = 0; u < U; u++)
                if (e + u * kTT < m) v[u] = __ldg(a + e + u * kTT);
#pragma unroll
            for (int u = 0; u < U; u++)
                if (e + u * kTT < m) w2[e + u * kTT] = v[u];
        }
    } else if (((uintptr_t)A & 15) == 0) {
        const float4 *a = static_cast<const float4 *>(A);
        const int64_t m = nn / 4;    // n even: n^2 is a multiple of 4
        for (int64_t e = tid; e < m; e += U * kTT) {
            float4 v[U];
#pragma unroll
            for (int u = 0; u < U; u++)
                if (e + u * kTT < m) v[u] = __ldg(a + e + u * kTT);
#pragma unroll
            for (int u = 0; u < U; u++)
                if (e + u * kTT < m) {
                    w2[2 * (e + u * kTT)] = make_double2(v[u].x, v[u].y);
                    w2[2 * (e + u * kTT) + 1] = make_double2(v[u].z, v[u].w);
                }
        }
    } else if (dt == PFB_F64) {
        const double *a = static_cast<const double *>(A);
        for (int64_t e = tid; e < nn; e += kTT) W[e] = a[e];
    } else {
        const float *a = static_cast<const float *>(A);
        for (int64_t e = tid; e < nn; e += kTT) W[e] = (double)a[e];
    }
}

template <int NB>
struct RaggedSmem {
    PanelSmem<double, NB> panel;
    alignas(16) double strip[NB][strip_ld<NB>()];   // the panel rows for the trailing update
    int item;
};

template <int NB>
__global__ void __launch_bounds__(kTT, RaggedCfg<NB>::kMinBlocks)
ragged_kernel(const void *const *__restrict__ As, const int32_t *__restrict__ ns,
              const int32_t *__restrict__ dts, int64_t count, int max_n, int layout,
              double *__restrict__ log_out, double *__restrict__ sign_out, unsigned char *__restrict__ ws,
              RaggedLayout L)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RaggedSmem<NB> &sm = *reinterpret_cast<RaggedSmem<NB> *>(smem_raw);
    const int32_t *order = reinterpret_cast<const int32_t *>(ws + L.order_off);
    int *counter = reinterpret_cast<int *>(ws + L.counter_off);
    unsigned char *mine = ws + L.cta_off + (size_t)blockIdx.x * L.cta_bytes;
    double *W = reinterpret_cast<double *>(mine + L.w_off);
    MatState *st = reinterpret_cast<MatState *>(mine + L.st_off);
    int32_t *piv = reinterpret_cast<int32_t *>(mine + L.piv_off);
    const int tid = threadIdx.x;

    for (;;) {
        if (tid == 0) {
            const int idx = atomicAdd(counter, 1);
            sm.item = idx < count ? order[idx] : -1;
        }
        __syncthreads();
        const int item = sm.item;
        __syncthreads();
        if (item < 0) break;
        const int n = ns[item];
        const int dt = dts[item];
        if (n < 0 || n > max_n || (dt != PFB_F32 && dt != PFB_F64)) {
            if (tid == 0) { log_out[item] = NAN; sign_out[item] = 0.0; }
            continue;
        }
        if (n == 0 || (n & 1)) {
            if (tid == 0) { log_out[item] = -INFINITY; sign_out[item] = 0.0; }
            continue;
        }
        // copy in (the row-major view; column-major input is its transpose -A)
        copy_in_item(W, As[item], dt, (int64_t)n * n);
        if (tid == 0) {
            MatState s0;
            s0.log_abs = 0.0;
            s0.ph_re = 1.0;
            s0.ph_im = 0.0;
            s0.parity = 0;
            s0.dead = 0;
            *st = s0;
        }
        __syncthreads();
        for (int k0 = 0; k0 < n - 1; k0 += NB) {
            panel_body<double, NB, kRaggedCPT, true>(sm.panel, W, n, k0, st, piv);
            if (st->dead) break;
            const int K = (n - k0 < NB) ? n - k0 : NB;
            cta_update<NB, RaggedCfg<NB>::kUpdBlock>(W, n, k0, K, sm.strip);
            __syncthreads();
        }
        if (tid == 0) {
            const MatState s = *st;
            if (s.dead) {
                log_out[item] = -INFINITY;
                sign_out[item] = 0.0;
            } else {
                const int neg = (s.parity ^ ((layout == PFB_COL_MAJOR) ? ((n >> 1) & 1) : 0)) & 1;
                log_out[item] = s.log_abs;
                sign_out[item] = neg ? -s.ph_re : s.ph_re;
            }
        }
        __syncthreads();
    }
}

template <int NB>
static int launch_ragged_nb(const void *const *A, const int32_t *n, const int32_t *dtype, int64_t count,
                            int max_n, int layout, double *log_out, double *sign_out, unsigned char *ws,
                            const RaggedLayout &L, cudaStream_t s)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int ctas = RaggedCfg<NB>::kMinBlocks * sms;
    if (ctas > kRaggedMaxCTAs) ctas = kRaggedMaxCTAs;
    if ((int64_t)ctas > count) ctas = (int)count;
    const size_t smem = sizeof(RaggedSmem<NB>);
    if (cudaFuncSetAttribute(ragged_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return PFB_ERR_CUDA;
    // launched as clusters of one CTA, the form the panel factorisation expects
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas, 1, 1);
    cfg.blockDim = dim3(kTT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, ragged_kernel<NB>, A, n, dtype, count, max_n, layout, log_out, sign_out, ws,
                           L) != cudaSuccess)
        return PFB_ERR_CUDA;
    return PFB_OK;
}

int launch_ragged(const void *const *A, const int32_t *n, const int32_t *dtype, int64_t count, int max_n,
                  int layout, double *log_out, double *sign_out, void *workspace, cudaStream_t s)
{
    const RaggedLayout L = ragged_layout(count, max_n);
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    ragged_order_kernel<<<1, 1024, 0, s>>>(n, count, reinterpret_cast<int32_t *>(ws + L.order_off),
                                          reinterpret_cast<int *>(ws + L.counter_off));
    if (launch_status() != PFB_OK) return PFB_ERR_CUDA;
    if (max_n <= RaggedCfg<16>::kMaxN)
        return launch_ragged_nb<16>(A, n, dtype, count, max_n, layout, log_out, sign_out, ws, L, s);
    return launch_ragged_nb<32>(A, n, dtype, count, max_n, layout, log_out, sign_out, ws, L, s);
}

}  // namespace pfb
