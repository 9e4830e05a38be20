// grad.cu -- the adjoint of log Pf: G = ct * d log Pf(A) / dA = ct * (1/2) A^-T,
// formed from the engine's own factorisation.
//
// The reference differentiates through JAX with jax.custom_jvp rules that call
// jnp.linalg.inv (pfcuda/cuda_api.py:78-107): d log Pf = (1/2) tr(A^-1 dA).
// Here the inverse comes from the blocked skew-LTL^T factors of large.cu:
//
//   P A P^T = U^T D U,   U block-unit upper triangular (2x2 identity blocks on
//   the diagonal), D = blockdiag(a_t J),  J = [[0, 1], [-1, 0]],
//
// where pair t contributes the rows U[2t] = w_t / a_t and U[2t+1] = u_t (the
// Gauss vectors the panel kernel stores as rows 2t+1 and 2t of W), and P is the
// product of the pivot interchanges.  Then
//
//   A^-1 = P^T Y D^-1 Y^T P,   Y = U^-1,   D^-1 = blockdiag(-J / a_t),
//
// so with Q[i][2t] = Y[i][2t+1] / a_t and Q[i][2t+1] = -Y[i][2t] / a_t,
// (P A^-1 P^T) = Q Y^T, and G[perm[r]][perm[c]] = -(ct/2) (Q Y^T)[r][c].
//
// Steps (all on the device, batched over matrices):
//   1. the forward factorisation (launch_large), which also yields (log, sign);
//   2. grad_fix_kernel: the interchanges of later panels are applied to the
//      Gauss vectors of earlier panels (the forward pass skips this), and the
//      permutation perm is built;
//   3. grad_diag_inv_kernel: the 64 x 64 diagonal blocks of Y = U^-1, in parallel;
//   4. grad_block_row_kernel, block rows from the bottom: Y_I,J>I = -Y_II (U_I,>I Y_>I,J);
//   5. grad_scatter_kernel: Q Y^T on the upper tiles, scaled and scattered to G.
// U is never stored: its entries are read from the Gauss vectors in W (u_entry).
//
// Memory budget: the workspace is the budget.  Per matrix the adjoint needs its
// working matrix W (the factors) and Y, about 2 n^2 elements; a workspace that
// holds fewer matrices than the batch makes the call run the batch in chunks of
// as many matrices as fit, each chunk factored, differentiated and its storage
// reused by the next.  Every matrix's arithmetic is independent of the others,
// so the results do not depend on the chunking.
#include "common.cuh"
#include "large.cuh"
#include "dmma.cuh"

namespace pfb {

constexpr int kGB = 64;   // block size of the triangular inverse and of the output tiles

struct GradLayout {
    size_t large_bytes, y_off, perm_off, total;
};

static size_t galign(size_t x) { return (x + 255) & ~(size_t)255; }

static GradLayout grad_layout(int dtype, int64_t B, int n, int mode)
{
    GradLayout L{};
    const size_t ts = (dtype == PFB_C64 || dtype == PFB_C128) ? 16 : 8;
    L.large_bytes = galign(large_workspace_bytes(dtype, B, n, mode));
    L.y_off = L.large_bytes;
    L.perm_off = galign(L.y_off + (size_t)B * n * n * ts);
    L.total = galign(L.perm_off + (size_t)B * n * sizeof(int32_t));
    return L;
}

size_t grad_workspace_bytes(int dtype, int64_t batch, int n, int mode)
{
    if (large_workspace_bytes(dtype, batch, n, mode) == 0) return 0;
    return grad_layout(dtype, batch, n, mode).total;
}

// 2. interchanges of later panels applied to earlier Gauss vectors; perm
template <typename T>
__global__ void grad_fix_kernel(T *__restrict__ W_all, const int32_t *__restrict__ piv_all,
                                int32_t *__restrict__ perm_all, const MatState *__restrict__ st_all, int n, int nb)
{
    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    T *W = W_all + b * (int64_t)n * n;
    const int32_t *piv = piv_all + b * (int64_t)(n / 2);
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) {
        // row r was written by the panel starting at (r / nb) * nb; the panels
        // after it interchanged columns it never saw
        for (int t = ((r / nb) + 1) * nb / 2; t < n / 2; t++) {
            const int i = 2 * t + 1, j = piv[t];
            if (j != i) {
                T *row = W + (int64_t)r * n;
                const T x = row[i];
                row[i] = row[j];
                row[j] = x;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int32_t *perm = perm_all + b * (int64_t)n;
        for (int q = 0; q < n; q++) perm[q] = q;
        for (int t = 0; t < n / 2; t++) {
            const int i = 2 * t + 1, j = piv[t];
            const int32_t x = perm[i];
            perm[i] = perm[j];
            perm[j] = x;
        }
    }
}

// Entry (r, c) of U (unit diagonal, zeros below it and at (2t, 2t+1)) from the
// Gauss vectors in W: row 2t+1 of U is u_t (row 2t of W), row 2t is w_t / a_t
// (row 2t+1 of W over the pivot W[2t][2t+1]); ia = 1 / a_t of row r's pair.
template <typename T>
PFB_D T u_entry(const T *__restrict__ W, int n, int r, int c, T ia)
{
    if (c == r) return one<T>();
    if (c <= (r | 1)) return zero<T>();
    const int t = r >> 1;
    return (r & 1) ? W[(int64_t)(2 * t) * n + c] : W[(int64_t)(2 * t + 1) * n + c] * ia;
}

// 3. Y_II = U_II^-1 for every diagonal block (zeros outside the block's upper part).
template <typename T>
__global__ void __launch_bounds__(kGB)
grad_diag_inv_kernel(const T *__restrict__ W_all, T *__restrict__ Y_all, const MatState *__restrict__ st_all, int n)
{
    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Us = reinterpret_cast<T *>(smem_raw);          // [kGB][kGB]
    T *Ys = Us + kGB * kGB;
    const T *W = W_all + b * (int64_t)n * n;
    T *Y = Y_all + b * (int64_t)n * n;
    const int r0 = blockIdx.x * kGB;
    const int sz = (n - r0) < kGB ? n - r0 : kGB;
    const int j = threadIdx.x;
    for (int i = 0; i < kGB; i++) {
        const int r = r0 + i;
        const T ia = (i < sz && !(r & 1)) ? recip(W[(int64_t)r * n + r + 1]) : zero<T>();
        Us[i * kGB + j] = (i < sz && j < sz) ? u_entry(W, n, r, r0 + j, ia) : zero<T>();
    }
    __syncthreads();
    // column j of the inverse by back substitution, one thread per column
    for (int i = kGB - 1; i >= 0; i--) {
        T v = zero<T>();
        if (i == j) {
            v = one<T>();
        } else if (i < j) {
            for (int k = i + 1; k <= j; k++) v = fms_(Us[i * kGB + k], Ys[k * kGB + j], v);
        }
        Ys[i * kGB + j] = v;
    }
    for (int i = 0; i < sz; i++)
        if (j < sz) Y[(int64_t)(r0 + i) * n + r0 + j] = Ys[i * kGB + j];
}

// Shared-memory row strides of the adjoint's DMMA tiles (dmma.cuh): a
// k-contiguous operand 32 (+4) or 64 (+4) wide, a k-major one 64 (+4 real,
// +2 complex) wide.
template <typename T> __host__ __device__ constexpr int ld_kc32() { return 36; }
template <typename T> __host__ __device__ constexpr int ld_kc64() { return 68; }
template <typename T> __host__ __device__ constexpr int ld_km64() { return IsComplex<T>::value ? 66 : 68; }

// 4. one block row I of Y (rows r0 .. r0+63), column tile blockIdx.x after it:
// Y[I][c] = -Y_II * sum_{k >= r1} U[I][k] Y[k][c], both products on the FP64
// tensor cores (8 warps, each a 32 x 16 block of m8n8k4 fragments).
template <typename T>
__global__ void __launch_bounds__(256)
grad_block_row_kernel(const T *__restrict__ W_all, T *__restrict__ Y_all, const MatState *__restrict__ st_all,
                      int n, int r0)
{
    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    constexpr int LA = ld_kc32<T>(), LB = ld_km64<T>(), LY = ld_kc64<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Ut = reinterpret_cast<T *>(smem_raw);        // [kGB][LA]  U[I][k]   (k-contiguous)
    T *Yt = Ut + kGB * LA;                           // [32][LB]   Y[k][c]   (k-major)
    T *Ts = reinterpret_cast<T *>(smem_raw);        // [kGB][LB]  the sum   (k-major), after the loop
    T *Yii = Ts + kGB * LB;                          // [kGB][LY]  Y_II      (k-contiguous)
    __shared__ T ias[kGB / 2];                       // 1 / a_t of the block row's pairs
    const T *W = W_all + b * (int64_t)n * n;
    T *Y = Y_all + b * (int64_t)n * n;
    if (threadIdx.x < kGB / 2) {
        const int r = r0 + 2 * threadIdx.x;
        ias[threadIdx.x] = r + 1 < n ? recip(W[(int64_t)r * n + r + 1]) : zero<T>();
    }
    __syncthreads();
    const int r1 = r0 + kGB;
    const int c0 = r1 + blockIdx.x * kGB;
    const int tid = threadIdx.x, warp = tid >> 5, g = (tid & 31) >> 2, t = tid & 3;
    const int wa = (warp >> 2) * 32, wb = (warp & 3) * 16;
    FragAcc<T, 4, 2> acc;
    acc.zero();
    const int kend = (c0 + kGB < n) ? c0 + kGB : n;    // Y[k][c] = 0 for k > c
    for (int k0 = r1; k0 < kend; k0 += 32) {
        for (int e = tid; e < kGB * 32; e += 256) {
            const int i = e / 32, k = e % 32;
            Ut[i * LA + k] = (r0 + i < n && k0 + k < n) ? u_entry(W, n, r0 + i, k0 + k, ias[i >> 1]) : zero<T>();
            const int kk = e / kGB, c = e % kGB;
            Yt[kk * LB + c] = (k0 + kk < n && c0 + c < n) ? Y[(int64_t)(k0 + kk) * n + c0 + c] : zero<T>();
        }
        __syncthreads();
#pragma unroll 1
        for (int kb = 0; kb < 32; kb += 4) acc.template step<false, true>(Ut + wa * LA, LA, Yt + wb, LB, kb);
        __syncthreads();
    }
    // the sum to shared memory (row = its k in the second product)
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int e2 = 0; e2 < 2; e2++) Ts[(wa + 8 * i + g) * LB + wb + 8 * j + 2 * t + e2] = acc.get(i, j, e2);
    for (int e = tid; e < kGB * kGB; e += 256) {
        const int i = e / kGB, k = e % kGB;
        Yii[i * LY + k] = (r0 + i < n && r0 + k < n) ? Y[(int64_t)(r0 + i) * n + r0 + k] : zero<T>();
    }
    __syncthreads();
    acc.zero();
#pragma unroll 1
    for (int kb = 0; kb < kGB; kb += 4) acc.template step<false, true>(Yii + wa * LY, LY, Ts + wb, LB, kb);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = r0 + wa + 8 * i + g;
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int e2 = 0; e2 < 2; e2++) {
                const int c = c0 + wb + 8 * j + 2 * t + e2;
                if (r < n && c < n) Y[(int64_t)r * n + c] = -acc.get(i, j, e2);
            }
    }
}

template <typename T>
constexpr size_t block_row_smem()
{
    constexpr size_t p1 = (size_t)(kGB * ld_kc32<T>() + 32 * ld_km64<T>()) * sizeof(T);
    constexpr size_t p2 = (size_t)(kGB * ld_km64<T>() + kGB * ld_kc64<T>()) * sizeof(T);
    return p1 > p2 ? p1 : p2;
}

template <typename T, typename O>
PFB_D O to_out(T v);
template <> PFB_D double to_out<double, double>(double v) { return v; }
template <> PFB_D float to_out<double, float>(double v) { return (float)v; }
template <> PFB_D c128 to_out<c128, c128>(c128 v) { return v; }
template <> PFB_D c64 to_out<c128, c64>(c128 v) { return mk((float)v.re, (float)v.im); }

// 5. M = Q Y^T on the upper 64 x 64 tiles, G[perm[r]][perm[c]] = -(ct/2) M[r][c]
// and its skew mirror, on the FP64 tensor cores.  Matrices with Pf = 0 get NaN.
template <typename T, typename O>
__global__ void __launch_bounds__(256)
grad_scatter_kernel(const T *__restrict__ W_all, const T *__restrict__ Y_all, const int32_t *__restrict__ perm_all,
                    const MatState *__restrict__ st_all, const double *__restrict__ ct, int n, O *__restrict__ G_all)
{
    const int64_t b = blockIdx.y;
    O *G = G_all + b * (int64_t)n * n;
    const int nt = (n + kGB - 1) / kGB;
    int L = blockIdx.x, I = 0;
    while (L >= nt - I) { L -= nt - I; I++; }
    const int J = I + L;
    const int i0 = I * kGB, j0 = J * kGB;
    const int tid = threadIdx.x;
    const int32_t *perm = perm_all + b * (int64_t)n;
    if (st_all[b].dead) {
        for (int e = tid; e < kGB * kGB; e += 256) {
            const int r = i0 + e / kGB, c = j0 + e % kGB;
            if (r < n && c < n) {
                T nanv;
                if constexpr (IsComplex<T>::value) nanv = mk((double)NAN, (double)NAN);
                else nanv = (T)NAN;
                G[(int64_t)r * n + c] = to_out<T, O>(nanv);
                G[(int64_t)c * n + r] = to_out<T, O>(nanv);
            }
        }
        return;
    }
    constexpr int LD = ld_kc32<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Qs = reinterpret_cast<T *>(smem_raw);       // [kGB][LD]  Q[i][k] for the tile's rows (k-contiguous)
    T *Ys = Qs + kGB * LD;                          // [kGB][LD]  Y[j][k] for the tile's columns
    T *ias = Ys + kGB * LD;                         // [16]       1 / a_t for the chunk's 16 pivot pairs
    const T *W = W_all + b * (int64_t)n * n;
    const T *Y = Y_all + b * (int64_t)n * n;
    const int warp = tid >> 5, g = (tid & 31) >> 2, t = tid & 3;
    const int wa = (warp >> 2) * 32, wb = (warp & 3) * 16;
    FragAcc<T, 4, 2> acc;
    acc.zero();
    for (int k0 = j0; k0 < n; k0 += 32) {            // Y[j][k] = 0 for k < j
        if (tid < 16) {
            const int p = (k0 >> 1) + tid;           // k0 is even
            ias[tid] = (2 * p + 1 < n) ? recip(W[(int64_t)(2 * p) * n + 2 * p + 1]) : zero<T>();
        }
        __syncthreads();
        for (int e = tid; e < 32 * kGB; e += 256) {
            const int x = e >> 5, k = e & 31;        // consecutive lanes: consecutive k of a row
            const int kg = k0 + k;
            T q = zero<T>(), y = zero<T>();
            if (kg < n) {
                if (i0 + x < n) {
                    const T ia = ias[k >> 1];
                    q = (kg & 1) ? (-Y[(int64_t)(i0 + x) * n + (kg - 1)]) * ia : Y[(int64_t)(i0 + x) * n + kg + 1] * ia;
                }
                if (j0 + x < n) y = Y[(int64_t)(j0 + x) * n + kg];
            }
            Qs[x * LD + k] = q;
            Ys[x * LD + k] = y;
        }
        __syncthreads();
#pragma unroll 1
        for (int kb = 0; kb < 32; kb += 4) acc.template step<false, false>(Qs + wa * LD, LD, Ys + wb * LD, LD, kb);
        __syncthreads();
    }
    const double s = -0.5 * (ct ? ct[b] : 1.0);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = i0 + wa + 8 * i + g;
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int e2 = 0; e2 < 2; e2++) {
                const int c = j0 + wb + 8 * j + 2 * t + e2;
                if (r < n && c < n && r <= c) {
                    const int pr = perm[r], pc = perm[c];
                    if (r == c) {
                        G[(int64_t)pr * n + pr] = to_out<T, O>(zero<T>());
                    } else {
                        const T gv = scal(acc.get(i, j, e2), s);
                        G[(int64_t)pr * n + pc] = to_out<T, O>(gv);
                        G[(int64_t)pc * n + pr] = to_out<T, O>(-gv);
                    }
                }
            }
    }
}

template <typename T>
constexpr size_t scatter_smem()
{
    return (size_t)(2 * kGB * ld_kc32<T>() + 16) * sizeof(T);
}

template <typename T>
static int run_grad(int dtype, const void *A, int64_t B, int n, int layout, int mode, const double *ct,
                    void *G, double *log_out, void *sign_out, unsigned char *ws, cudaStream_t s)
{
    const GradLayout L = grad_layout(dtype, B, n, mode);
    int rc = launch_large(dtype, A, B, n, layout, mode, log_out, sign_out, ws, L.large_bytes, s, nullptr);
    if (rc != PFB_OK) return rc;
    const LargeView V = large_view(dtype, B, n, mode, ws);
    T *W = static_cast<T *>(V.W);
    T *Y = reinterpret_cast<T *>(ws + L.y_off);
    int32_t *perm = reinterpret_cast<int32_t *>(ws + L.perm_off);
    const int nb = large_panel_width(dtype, n);
    const unsigned ub = (unsigned)B;

    grad_fix_kernel<T><<<dim3((n + 255) / 256, ub), 256, 0, s>>>(W, V.piv, perm, V.st, n, nb);
    const int nblk = (n + kGB - 1) / kGB;
    {
        auto k = grad_diag_inv_kernel<T>;
        const size_t sm = 2 * kGB * kGB * sizeof(T);
        if (cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) != PFB_OK) return PFB_ERR_CUDA;
        k<<<dim3((unsigned)nblk, ub), kGB, sm, s>>>(W, Y, V.st, n);
    }
    {
        auto k = grad_block_row_kernel<T>;
        const size_t sm = block_row_smem<T>();
        if (cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) != PFB_OK) return PFB_ERR_CUDA;
        for (int I = nblk - 2; I >= 0; I--) {
            const int r0 = I * kGB;
            const int tiles = (n - (r0 + kGB) + kGB - 1) / kGB;
            k<<<dim3((unsigned)tiles, ub), 256, sm, s>>>(W, Y, V.st, n, r0);
        }
    }
    {
        const unsigned tiles = (unsigned)(nblk * (nblk + 1) / 2);
        const size_t sm = (dtype == PFB_C64 || dtype == PFB_C128) ? scatter_smem<c128>() : scatter_smem<double>();
        if (dtype == PFB_F32) {
            auto k = grad_scatter_kernel<double, float>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k<<<dim3(tiles, ub), 256, sm, s>>>((const double *)W, (const double *)Y, perm, V.st, ct, n, (float *)G);
        } else if (dtype == PFB_F64) {
            auto k = grad_scatter_kernel<double, double>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k<<<dim3(tiles, ub), 256, sm, s>>>((const double *)W, (const double *)Y, perm, V.st, ct, n, (double *)G);
        } else if (dtype == PFB_C64) {
            auto k = grad_scatter_kernel<c128, c64>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k<<<dim3(tiles, ub), 256, sm, s>>>((const c128 *)W, (const c128 *)Y, perm, V.st, ct, n, (c64 *)G);
        } else {
            auto k = grad_scatter_kernel<c128, c128>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k<<<dim3(tiles, ub), 256, sm, s>>>((const c128 *)W, (const c128 *)Y, perm, V.st, ct, n, (c128 *)G);
        }
    }
    return launch_status();
}

// The largest number of matrices (<= batch) whose adjoint fits in `bytes` of
// workspace; 0 if not even one does.
int64_t grad_chunk(int dtype, int64_t batch, int n, int mode, size_t bytes)
{
    if (grad_workspace_bytes(dtype, 1, n, mode) > bytes) return 0;
    int64_t lo = 1, hi = batch;
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo + 1) / 2;
        if (grad_workspace_bytes(dtype, mid, n, mode) <= bytes) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

int launch_grad(int dtype, const void *A, int64_t batch, int n, int layout, int mode, const double *ct, void *G,
                double *log_out, void *sign_out, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    const int64_t chunk = grad_chunk(dtype, batch, n, mode, workspace_bytes);
    if (chunk <= 0) return PFB_ERR_WORKSPACE;
    const size_t es = (dtype == PFB_F32) ? 4 : (dtype == PFB_C128 ? 16 : 8);
    const size_t mat = (size_t)n * (size_t)n * es;
    for (int64_t b0 = 0; b0 < batch; b0 += chunk) {
        const int64_t B = batch - b0 < chunk ? batch - b0 : chunk;
        const void *a = static_cast<const char *>(A) + (size_t)b0 * mat;
        void *g = static_cast<char *>(G) + (size_t)b0 * mat;
        void *so = static_cast<char *>(sign_out) + (size_t)b0 * es;
        const double *c = ct ? ct + b0 : nullptr;
        const int rc = (dtype == PFB_C64 || dtype == PFB_C128)
                           ? run_grad<c128>(dtype, a, B, n, layout, mode, c, g, log_out + b0, so, ws, stream)
                           : run_grad<double>(dtype, a, B, n, layout, mode, c, g, log_out + b0, so, ws, stream);
        if (rc != PFB_OK) return rc;
    }
    return PFB_OK;
}

}  // namespace pfb
