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
//   * copy_in: the input (any dtype, either layout) becomes an FP64 / complex128
//     working matrix W in the workspace, row-major, of which only the strict
//     upper triangle is read from then on.
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
//     (w, -u) -- a skew rank-NB update, FP64 here (gemm_fp64_kernel) or
//     error-free int8 slices on the tcgen05 tensor cores (split.cu).
//   * finalize: log/sign from the per-matrix state.
// Column-major input is handled like the small path: its row-major view is the
// transpose -A, and Pf(-A) = (-1)^(n/2) Pf(A) exactly.
#include <limits.h>

#include "common.cuh"
#include "large.cuh"
#include "split.cuh"

namespace pfb {

constexpr int kTT = 256;         // trailing-column threads per CTA
constexpr int kClusterMax = 16;  // non-portable cluster size limit

// --------------------------------------------------------------- PTX helpers

PFB_D uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
PFB_D uint32_t cluster_size()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
PFB_D void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release;\n\t"
                 "barrier.cluster.wait.acquire;" ::: "memory");
}
PFB_D uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
PFB_D uint32_t map_rank(uint32_t addr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
PFB_D void st_remote(uint32_t addr, double v)
{
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
PFB_D void st_remote(uint32_t addr, int v)
{
    asm volatile("st.shared::cluster.s32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
PFB_D void st_remote(uint32_t addr, c128 v)
{
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.re), "d"(v.im) : "memory");
}
// L2-coherent accesses to the working matrix inside the panel kernel: other
// CTAs of the cluster read and write the same lines between cluster barriers.
PFB_D double ldcg(const double *p) { return __ldcg(p); }
PFB_D c128 ldcg(const c128 *p)
{
    double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return mk(v.x, v.y);
}
PFB_D void stcg(double *p, double v) { __stcg(p, v); }
PFB_D void stcg(c128 *p, c128 v) { __stcg(reinterpret_cast<double2 *>(p), make_double2(v.re, v.im)); }

PFB_D double pkey(double x)
{
    double m = fabs(x);
    return (m != m) ? INFINITY : m;
}
PFB_D double pkey(c128 x)
{
    double m = hypot(x.re, x.im);
    return (m != m) ? INFINITY : m;
}
PFB_D c128 neg(c128 x) { return mk(-x.re, -x.im); }
PFB_D double neg(double x) { return -x; }

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

size_t large_workspace_bytes(int dtype, int64_t batch, int n, int mode)
{
    int nb, cpt;
    if (n > 32 && !large_cfg(dtype, n, &nb, &cpt)) return 0;
    return large_layout(dtype, batch, n, mode).total;
}

// ----------------------------------------------------------------- copy in

template <typename S, typename T>
__global__ void copy_in_kernel(const S *__restrict__ A, T *__restrict__ W, int64_t total,
                               MatState *st, int64_t batch)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride)
        W[e] = conv<T>(A[e]);
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

// ----------------------------------------------------------------- panel

template <typename T, int NB>
struct PanelSmem {
    using Real = typename RealOf<T>::type;
    static constexpr int NT = kTT;
    static constexpr int NW = NT / 32;
    T lb[NB][NB + 1];                  // replicated NB x NB block of the panel columns
    alignas(16) T stage[2][NB];        // this CTA's best trailing column, panel rows 0..NB-1
    T hval[2][kClusterMax];            // per-CTA best candidate, pushed by every CTA of the cluster
    Real hkey[2][kClusterMax];
    int hcol[2][kClusterMax];
    T wval[NW];                        // per-warp best candidate
    Real wkey[NW];
    int wcol[NW];
    T pivval[NB / 2];                  // this panel's pivots and pivot columns
    int pivcol[NB / 2];
};

template <typename T> PFB_D void put(uint32_t a, T v) { st_remote(a, v); }
PFB_D void store_pair(double *p, double a, double b) { *reinterpret_cast<double2 *>(p) = make_double2(a, b); }
PFB_D void store_pair(c128 *p, c128 a, c128 b) { p[0] = a; p[1] = b; }

// s + sum over the window's Gauss-vector pairs (window pair index P >= fin0,
// pair u = P - fin0) of  c_u[u] * Rw[2P+1] - c_w[u] * Rw[2P]  with
// c_u = lb[2u][col], c_w = lb[2u+1][col].  Four partial sums shorten the
// dependency chain; chunks of 8 pairs with a compiler barrier between them keep
// the coefficient loads from all being hoisted into registers at once.
template <typename T, int NB>
PFB_D T lazy_row(T s, const T (&Rw)[NB], const T (*lb)[NB + 1], int col, int fin0)
{
    T s2 = zero<T>(), s3 = zero<T>(), s4 = zero<T>();
#pragma unroll
    for (int P0 = 0; P0 < NB / 2; P0 += 8) {
        if (P0 + 7 >= fin0) {
#pragma unroll
            for (int P = P0; P < P0 + 8; P++) {
                if (P >= 1 && P >= fin0) {
                    const int u = P - fin0;
                    if (P & 1) {
                        s = fma_(lb[2 * u][col], Rw[2 * P + 1], s);
                        s2 = fms_(lb[2 * u + 1][col], Rw[2 * P], s2);
                    } else {
                        s3 = fma_(lb[2 * u][col], Rw[2 * P + 1], s3);
                        s4 = fms_(lb[2 * u + 1][col], Rw[2 * P], s4);
                    }
                }
            }
        }
        asm volatile("" ::: "memory");
    }
    return (s + s2) + (s3 + s4);
}

// Interchange window rows 1 and p (2 <= p < NB, uniform across the CTA) with
// a branch per position, so every register index stays static.
template <typename T, int NB>
PFB_D void swap_window_row(T (&Rw)[NB], int p)
{
    static_for<2, NB, 1>([&](auto pc) {
        constexpr int P = decltype(pc)::value;
        if (p == P) {
            const T tmp = Rw[1];
            Rw[1] = Rw[P];
            Rw[P] = tmp;
        }
    });
}

PFB_D double ld_remote(uint32_t addr, double *)
{
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
    return v;
}
PFB_D c128 ld_remote(uint32_t addr, c128 *)
{
    double re, im;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(re), "=d"(im) : "r"(addr) : "memory");
    return mk(re, im);
}

// Factor panel rows [k0, k0+NB) of every matrix; one cluster of CL CTAs per
// matrix (blockIdx.y).  Thread i of CTA rank r keeps trailing columns
// k0+NB + r*kTT + i + q*CL*kTT (q < CPT) of the panel rows in registers; threads
// i < NB also own panel column k0+i, whose entries live in the shared block lb.
//
// The register window is rotated by two rows per pivot step, so the current
// pivot rows are always Rw[0] (row k) and Rw[1] (row k+1) and the step loop
// stays a loop (a fully unrolled panel does not fit the instruction cache).  At
// step t, window position p holds panel row 2t+p for p < NB-2t (rows not yet
// factored) and panel row p-(NB-2t) otherwise (the Gauss vectors of pairs
// 0..t-1, u_s at even and w_s at odd positions).
//
// A pivot step costs one cluster barrier: every CTA pushes the header of its
// best candidate (|value|, column, value) into every CTA's shared memory before
// it, and the owner of a CTA's best trailing column stages that column; after
// the barrier each CTA knows the pivot, and the panel-column threads read the
// interchanged column straight from the winning CTA's stage.
template <typename T, int NB, int CPT>
__global__ void __launch_bounds__(kTT, 1)
panel_kernel(T *__restrict__ W_all, int n, int k0, MatState *__restrict__ st_all,
             int32_t *__restrict__ piv_all, SplitArgs split)
{
    using Real = typename RealOf<T>::type;
    using SM = PanelSmem<T, NB>;
    constexpr int NW = SM::NW;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM &sm = *reinterpret_cast<SM *>(smem_raw);

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const bool has_panel = tid < NB;
    const uint32_t rank = cluster_rank();
    const int CL = (int)cluster_size();
    const int64_t b = blockIdx.y;
    T *W = W_all + b * (int64_t)n * n;
    MatState *st = st_all + b;
    int32_t *piv = piv_all + b * (int64_t)(n / 2);

    if (st->dead) return;   // same value for the whole cluster

    const int k1 = k0 + NB;
    const int GT = CL * kTT;
    const int pc = k0 + tid;   // panel column of this thread (if has_panel)
    int cq[CPT];
#pragma unroll
    for (int q = 0; q < CPT; q++) cq[q] = k1 + (int)rank * kTT + tid + q * GT;

    // ---- load the panel rows (window position p = panel row p at step 0)
    T Rw[CPT][NB];
#pragma unroll
    for (int q = 0; q < CPT; q++)
#pragma unroll
        for (int r = 0; r < NB; r++)
            Rw[q][r] = (cq[q] < n && k0 + r < n) ? W[(int64_t)(k0 + r) * n + cq[q]] : zero<T>();
    if (has_panel) {
        for (int r = 0; r < NB; r++)
            sm.lb[r][tid] = (k0 + r < n && pc < n) ? W[(int64_t)(k0 + r) * n + pc] : zero<T>();
    }

    double la = 0.0, pre = 1.0, pim = 0.0;
    int parity = 0;
    const bool leader = rank == 0 && tid == 0;
    if (leader) {
        la = st->log_abs;
        pre = st->ph_re;
        pim = st->ph_im;
        parity = st->parity;
    }
    bool dead = false;
    const int nsteps = (n - k0) / 2 < NB / 2 ? (n - k0) / 2 : NB / 2;
    // every CTA of the cluster has started (and loaded) before any shared
    // memory of another CTA is written
    cluster_sync();

    int t = 0;
#pragma unroll 1
    for (; t < nsteps; t++) {
        const int k = k0 + 2 * t;
        const int par = t & 1;
        const int fin0 = NB / 2 - t;   // window pair index of the oldest Gauss-vector pair

        // (1) lazy update of row k with the panel's earlier Gauss vectors
#pragma unroll
        for (int q = 0; q < CPT; q++) Rw[q][0] = lazy_row<T, NB>(Rw[q][0], Rw[q], sm.lb, 2 * t, fin0);
        const bool pcand = has_panel && tid > 2 * t && pc < n;
        T pv = zero<T>();
        if (pcand) {
            T s = sm.lb[2 * t][tid];
            for (int u = 0; u < t; u++) {
                s = fma_(sm.lb[2 * u][2 * t], sm.lb[2 * u + 1][tid], s);
                s = fms_(sm.lb[2 * u + 1][2 * t], sm.lb[2 * u][tid], s);
            }
            sm.lb[2 * t][tid] = s;
            pv = s;
        }

        // (2) this thread's best candidate (its panel column first: the
        // smaller index), then the warp's
        Real key = (Real)(-1);
        int col = INT_MAX;
        int qsel = -1;
        T val = zero<T>();
        if (pcand) { key = pkey(pv); col = pc; val = pv; }
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            if (cq[q] < n) {
                Real kq = pkey(Rw[q][0]);
                if (kq > key) { key = kq; col = cq[q]; qsel = q; val = Rw[q][0]; }
            }
        }
        Real wk = key;
        int wc = col;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            Real k2 = shfl_xor(wk, off);
            int c2 = shfl_xor(wc, off);
            if (k2 > wk || (k2 == wk && c2 < wc)) { wk = k2; wc = c2; }
        }
        if (wc != INT_MAX && col == wc) sm.wval[warp] = val;
        if (lane == 0) { sm.wkey[warp] = wk; sm.wcol[warp] = wc; }
        __syncthreads();

        // (3) the CTA's best candidate: its header goes to every CTA of the
        // cluster, and if it is a trailing column its owner stages the column
        Real ck = (Real)(-1);
        int cc = INT_MAX, cw = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            Real kk = sm.wkey[w];
            int c = sm.wcol[w];
            if (kk > ck || (kk == ck && c < cc)) { ck = kk; cc = c; cw = w; }
        }
        if (tid < CL) {
            put(map_rank(smem_u32(&sm.hkey[par][rank]), tid), ck);
            put(map_rank(smem_u32(&sm.hcol[par][rank]), tid), cc);
            put(map_rank(smem_u32(&sm.hval[par][rank]), tid), sm.wval[cw]);
        }
        if (qsel >= 0 && col == cc) {
#pragma unroll
            for (int P = 0; P < NB / 2; P++) {
                // window pair P holds panel rows (r, r+1), r even
                const int r = (2 * P < NB - 2 * t) ? 2 * t + 2 * P : 2 * P - (NB - 2 * t);
                T v0 = Rw[0][2 * P], v1 = Rw[0][2 * P + 1];
#pragma unroll
                for (int q = 1; q < CPT; q++) {
                    v0 = (qsel == q) ? Rw[q][2 * P] : v0;
                    v1 = (qsel == q) ? Rw[q][2 * P + 1] : v1;
                }
                store_pair(&sm.stage[par][r], v0, v1);
            }
        }
        cluster_sync();

        // (4) the pivot: a tree over the CL headers
        Real hk[kClusterMax];
        int hc[kClusterMax], hs[kClusterMax];
#pragma unroll
        for (int s2 = 0; s2 < kClusterMax; s2++) {
            hk[s2] = s2 < CL ? sm.hkey[par][s2] : (Real)(-1);
            hc[s2] = s2 < CL ? sm.hcol[par][s2] : INT_MAX;
            hs[s2] = s2;
        }
#pragma unroll
        for (int w = kClusterMax / 2; w > 0; w >>= 1) {
#pragma unroll
            for (int s2 = 0; s2 < w; s2++) {
                if (hk[s2 + w] > hk[s2] || (hk[s2 + w] == hk[s2] && hc[s2 + w] < hc[s2])) {
                    hk[s2] = hk[s2 + w];
                    hc[s2] = hc[s2 + w];
                    hs[s2] = hs[s2 + w];
                }
            }
        }
        const int j = hc[0], gs = hs[0];
        const T a = sm.hval[par][gs];
        if (is_zero(a) || j == INT_MAX) { dead = true; break; }

        // (5) interchange k+1 <-> j on the upper triangle.  The trailing rows'
        // entries come from global memory; their loads are issued here and
        // consumed after the barriers below, so their latency overlaps them.
        T gl[CPT];
        bool gneg[CPT], guse[CPT];
#pragma unroll
        for (int q = 0; q < CPT; q++) { gl[q] = zero<T>(); gneg[q] = false; guse[q] = false; }
        if (j != k + 1) {
            const int jl = j - k0;
            const bool trail_win = j >= k1;
            T tI = zero<T>(), tJ = zero<T>(), tRi = zero<T>(), tRj = zero<T>();
            if (!trail_win) {
                // rows k+1 (position 1) and j (position jl - 2t) of every trailing column
#pragma unroll
                for (int q = 0; q < CPT; q++) swap_window_row<T, NB>(Rw[q], jl - 2 * t);
                if (has_panel) {
                    const int x = tid;
                    if (x <= 2 * t) { tI = sm.lb[x][2 * t + 1]; tJ = sm.lb[x][jl]; }
                    if (x > 2 * t + 1 && x < jl) { tJ = sm.lb[x][jl]; tRi = sm.lb[2 * t + 1][x]; }
                    if (x == jl) tRi = sm.lb[2 * t + 1][jl];
                    if (x > jl) { tRi = sm.lb[2 * t + 1][x]; tRj = sm.lb[jl][x]; }
                }
            } else {
#pragma unroll
                for (int q = 0; q < CPT; q++) {
                    const int c = cq[q];
                    if (c == j) {
                        // the new column j: rows < k+1 from column k+1, (k+1, j) negated,
                        // rows > k+1 from row k+1 negated
#pragma unroll
                        for (int p = 0; p < NB; p++) {
                            const int r = (p < NB - 2 * t) ? 2 * t + p : p - (NB - 2 * t);
                            if (p == 1) Rw[q][1] = neg(Rw[q][1]);
                            else if (r <= 2 * t) Rw[q][p] = sm.lb[r][2 * t + 1];
                            else Rw[q][p] = neg(sm.lb[2 * t + 1][r]);
                        }
                    } else if (c < n) {
                        const T old = Rw[q][1];
                        T *pp = (c < j) ? &W[(int64_t)c * n + j] : &W[(int64_t)j * n + c];
                        gl[q] = ldcg(pp);
                        gneg[q] = c < j;
                        guse[q] = true;
                        stcg(pp, c < j ? neg(old) : old);
                    }
                }
                if (has_panel)
                    tJ = ld_remote(map_rank(smem_u32(&sm.stage[par][tid]), (uint32_t)gs), (T *)nullptr);
            }
            __syncthreads();
            if (has_panel) {
                const int x = tid;
                if (!trail_win) {
                    if (x <= 2 * t) { sm.lb[x][2 * t + 1] = tJ; sm.lb[x][jl] = tI; }
                    if (x > 2 * t + 1 && x < jl) { sm.lb[2 * t + 1][x] = neg(tJ); sm.lb[x][jl] = neg(tRi); }
                    if (x == jl) sm.lb[2 * t + 1][jl] = neg(tRi);
                    if (x > jl) { sm.lb[2 * t + 1][x] = tRj; sm.lb[jl][x] = tRi; }
                } else {
                    if (x <= 2 * t) sm.lb[x][2 * t + 1] = tJ;
                    if (x > 2 * t + 1) sm.lb[2 * t + 1][x] = neg(tJ);
                }
            }
            __syncthreads();
            parity ^= 1;
        }
#pragma unroll
        for (int q = 0; q < CPT; q++)
            if (guse[q]) Rw[q][1] = gneg[q] ? neg(gl[q]) : gl[q];

        // (6) lazy update of row k+1, then u = row_k / a, w = -row_{k+1}
        const T ia = recip(a);
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            Rw[q][1] = neg(lazy_row<T, NB>(Rw[q][1], Rw[q], sm.lb, 2 * t + 1, fin0));
            Rw[q][0] = Rw[q][0] * ia;
        }
        if (has_panel && tid > 2 * t + 1 && pc < n) {
            T s = sm.lb[2 * t + 1][tid];
            for (int u = 0; u < t; u++) {
                s = fma_(sm.lb[2 * u][2 * t + 1], sm.lb[2 * u + 1][tid], s);
                s = fms_(sm.lb[2 * u + 1][2 * t + 1], sm.lb[2 * u][tid], s);
            }
            sm.lb[2 * t + 1][tid] = neg(s);
            sm.lb[2 * t][tid] = sm.lb[2 * t][tid] * ia;
        }
        if (tid == 0) {
            sm.pivval[t] = a;
            sm.pivcol[t] = j;
        }

        // (7) rotate the window: the finished pair goes to the end
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const T r0 = Rw[q][0], r1 = Rw[q][1];
#pragma unroll
            for (int p = 0; p < NB - 2; p++) Rw[q][p] = Rw[q][p + 2];
            Rw[q][NB - 2] = r0;
            Rw[q][NB - 1] = r1;
        }
        __syncthreads();
    }

    if (dead) {
        if (leader) st->dead = 1;
        cluster_sync();
        return;
    }
    if (leader) {
        for (int s2 = 0; s2 < t; s2++) {
            const T a = sm.pivval[s2];
            piv[k0 / 2 + s2] = sm.pivcol[s2];
            const double m = (double)mag(a);
            la += log(m);
            double ar, ai;
            if constexpr (IsComplex<T>::value) { ar = a.re / m; ai = a.im / m; }
            else { ar = a < 0 ? -1.0 : 1.0; ai = 0.0; }
            const double nr = pre * ar - pim * ai, ni = pre * ai + pim * ar;
            pre = nr;
            pim = ni;
        }
    }

    // ---- write the factored panel rows back (t steps done: window position p
    // holds panel row 2t+p for p < NB-2t, else row p-(NB-2t))
#pragma unroll
    for (int q = 0; q < CPT; q++)
#pragma unroll
        for (int p = 0; p < NB; p++) {
            const int r = (p < NB - 2 * t) ? 2 * t + p : p - (NB - 2 * t);
            if (cq[q] < n && k0 + r < n) W[(int64_t)(k0 + r) * n + cq[q]] = Rw[q][p];
        }
    if (has_panel && rank == 0 && pc < n) {
        for (int r = 0; r < NB && r < tid; r++) W[(int64_t)(k0 + r) * n + pc] = sm.lb[r][tid];
    }
    // the int8 operands of the split update; trailing columns exist only when
    // the panel is full (t == NB/2), where the window is back in row order
    if (split.enabled && t == NB / 2) {
#pragma unroll
        for (int q = 0; q < CPT; q++)
            if (cq[q] < n) split_panel_column<T, NB>(split, b, cq[q] - k1, Rw[q], NB);
    }
    if (leader) {
        // keep the phase on the unit circle across panels
        const double m = sqrt(pre * pre + pim * pim);
        st->log_abs = la;
        st->ph_re = pre / m;
        st->ph_im = pim / m;
        st->parity = parity;
    }
    cluster_sync();
}

// ------------------------------------------------------- FP64 trailing update

// S22[a][b] += sum_t X[t][a] * Y[t][b] over the upper-triangle tiles of the
// trailing block [k1, n), X = panel rows k0..k0+K-1, Y[2s] = X[2s+1],
// Y[2s+1] = -X[2s].  A BM x BN tile per 256-thread block, K <= KMAX in one
// shared-memory stage, TM x TN outputs per thread.
template <typename T, int BM, int BN, int KMAX, int TM, int TN>
__global__ void __launch_bounds__(256)
gemm_fp64_kernel(T *__restrict__ W_all, int n, int k0, int K, const MatState *__restrict__ st_all)
{
    static_assert((BM / TM) * (BN / TN) == 256, "thread tile");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Xs = reinterpret_cast<T *>(smem_raw);            // [KMAX][BM]
    T *Ys = Xs + KMAX * BM;                              // [KMAX][BN]
    const int64_t b = blockIdx.y;
    if (st_all[b].dead) return;
    T *W = W_all + b * (int64_t)n * n;
    const int k1 = k0 + K;
    const int m = n - k1;
    const int nt = (m + BM - 1) / BM;   // BM == BN
    // upper-triangle tile (I, J), J >= I, from the linear block index
    int L = blockIdx.x, I = 0;
    while (L >= nt - I) { L -= nt - I; I++; }
    const int J = I + L;
    const int a0 = k1 + I * BM, b0 = k1 + J * BN;
    const int tid = threadIdx.x;

    for (int e = tid; e < K * BM; e += 256) {
        const int r = e / BM, x = e - r * BM;
        Xs[r * BM + x] = (a0 + x < n) ? W[(int64_t)(k0 + r) * n + a0 + x] : zero<T>();
    }
    for (int e = tid; e < K * BN; e += 256) {
        const int r = e / BN, y = e - r * BN;
        T v = zero<T>();
        if (b0 + y < n) {
            const T s = W[(int64_t)(k0 + (r ^ 1)) * n + b0 + y];
            v = (r & 1) ? neg(s) : s;
        }
        Ys[r * BN + y] = v;
    }
    __syncthreads();

    const int tx = tid % (BN / TN), ty = tid / (BN / TN);
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int jj = 0; jj < TN; jj++) acc[i][jj] = zero<T>();

    for (int r = 0; r < K; r++) {
        T xa[TM], yb[TN];
#pragma unroll
        for (int i = 0; i < TM; i++) xa[i] = Xs[r * BM + ty + i * (BM / TM)];
#pragma unroll
        for (int jj = 0; jj < TN; jj++) yb[jj] = Ys[r * BN + tx + jj * (BN / TN)];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int jj = 0; jj < TN; jj++) acc[i][jj] = fma_(xa[i], yb[jj], acc[i][jj]);
    }
    // per output row: all loads first, then the stores (one memory round trip per row)
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int ar = a0 + ty + i * (BM / TM);
        if (ar >= n) continue;
        T cv[TN];
#pragma unroll
        for (int jj = 0; jj < TN; jj++) {
            const int bc = b0 + tx + jj * (BN / TN);
            cv[jj] = (bc < n && bc > ar) ? W[(int64_t)ar * n + bc] : zero<T>();
        }
#pragma unroll
        for (int jj = 0; jj < TN; jj++) {
            const int bc = b0 + tx + jj * (BN / TN);
            if (bc < n && bc > ar) W[(int64_t)ar * n + bc] = cv[jj] + acc[i][jj];
        }
    }
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
static int run_large(const void *A, int dtype, int64_t B, int n, int layout, int mode,
                     double *log_out, void *sign_out, unsigned char *ws, cudaStream_t s,
                     const pfb_slog_timing *tm)
{
    using SM = PanelSmem<T, NB>;
    const LargeLayout L = large_layout(dtype, B, n, mode);
    int32_t *piv = reinterpret_cast<int32_t *>(ws + L.piv_off);
    MatState *st = reinterpret_cast<MatState *>(ws + L.st_off);
    T *W = reinterpret_cast<T *>(ws + L.w_off);
    const int64_t total = B * (int64_t)n * n;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    {
        int64_t blocks = (total + 255) / 256;
        if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
        if (blocks < 1) blocks = 1;
        switch (dtype) {
        case PFB_F32:
            copy_in_kernel<float, double><<<(unsigned)blocks, 256, 0, s>>>(
                (const float *)A, (double *)W, total, st, B);
            break;
        case PFB_F64:
            copy_in_kernel<double, double><<<(unsigned)blocks, 256, 0, s>>>(
                (const double *)A, (double *)W, total, st, B);
            break;
        case PFB_C64:
            copy_in_kernel<c64, c128><<<(unsigned)blocks, 256, 0, s>>>(
                (const c64 *)A, (c128 *)W, total, st, B);
            break;
        default:
            copy_in_kernel<c128, c128><<<(unsigned)blocks, 256, 0, s>>>(
                (const c128 *)A, (c128 *)W, total, st, B);
            break;
        }
        if (cudaGetLastError() != cudaSuccess) return PFB_ERR_CUDA;
    }

    auto pk = panel_kernel<T, NB, CPT>;
    const size_t psmem = sizeof(SM);
    if (cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem) != cudaSuccess)
        return PFB_ERR_CUDA;
    if (cudaFuncSetAttribute(pk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return PFB_ERR_CUDA;

    constexpr bool cplx = IsComplex<T>::value;
    constexpr int BM = cplx ? 64 : 128;
    constexpr int TM = cplx ? 4 : 8;
    auto gk = gemm_fp64_kernel<T, BM, BM, NB, TM, TM>;
    const size_t gsmem = (size_t)2 * NB * BM * sizeof(T);
    if (cudaFuncSetAttribute(gk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem) != cudaSuccess)
        return PFB_ERR_CUDA;

    SplitArgs sa{};
    unsigned char *split_ws = ws + L.split_off;
    const int slices = ((mode >> 8) & 0xf) ? ((mode >> 8) & 0xf) : kSplitDefaultSlices;
    int32_t *split_err = nullptr;
    if ((mode & 0xff) == PFB_MODE_SPLIT) {
        split_err = split_args(true, split_ws, cplx, B, n, NB, 0, slices).err;
        if (cudaMemsetAsync(split_err, 0, (size_t)B * sizeof(int32_t), s) != cudaSuccess) return PFB_ERR_CUDA;
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
        sa = split_args(use_split, split_ws, cplx, B, n, NB, k0, slices);

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
        if (cudaLaunchKernelEx(&cfg, pk, W, n, k0, st, piv, sa) != cudaSuccess) return PFB_ERR_CUDA;
        rec(tm ? tm->panel_events : nullptr, 2 * panel_idx + 1);

        if (mt > 0) {
            rec(tm ? tm->update_events : nullptr, 2 * panel_idx);
            if (use_split) {
                int rc = launch_split_update(cplx, W, n, k0, K, B, st, sa, s);
                if (rc != PFB_OK) return rc;
            } else {
                const int nt = (mt + BM - 1) / BM;
                const unsigned tiles = (unsigned)(nt * (nt + 1) / 2);
                gk<<<dim3(tiles, (unsigned)B), 256, gsmem, s>>>(W, n, k0, K, st);
                if (cudaGetLastError() != cudaSuccess) return PFB_ERR_CUDA;
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
    return cudaGetLastError() == cudaSuccess ? PFB_OK : PFB_ERR_CUDA;
}

int launch_large(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                 double *log_out, void *sign_out, void *workspace, size_t workspace_bytes,
                 cudaStream_t stream, const pfb_slog_timing *timing)
{
    int nb = 0, cpt = 0;
    if (!large_cfg(dtype, n, &nb, &cpt)) return PFB_ERR_SIZE;
    if ((mode & 0xff) == PFB_MODE_SPLIT && !split_available()) return PFB_ERR_UNSUPPORTED;
    if (batch > 65535) return PFB_ERR_SIZE;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    const bool cplx = dtype == PFB_C64 || dtype == PFB_C128;
    if (!cplx) {
        if (nb == 64) return run_large<double, 64, 1>(A, dtype, batch, n, layout, mode, log_out, sign_out, ws, stream, timing);
        return run_large<double, 32, 2>(A, dtype, batch, n, layout, mode, log_out, sign_out, ws, stream, timing);
    }
    return run_large<c128, 32, 1>(A, dtype, batch, n, layout, mode, log_out, sign_out, ws, stream, timing);
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
