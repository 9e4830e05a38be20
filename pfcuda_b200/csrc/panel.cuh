// panel.cuh -- the panel factorisation of the blocked skew-LTL^T (see large.cu
// for the whole algorithm): one cluster of CTAs (or one CTA) factors NB pivot
// rows of one matrix, with the Gauss vectors of each trailing column in the
// registers of one thread.
#pragma once
#include <limits.h>

#include "common.cuh"
#include "large.cuh"

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
// The panel's barrier: the cluster barrier, or for a panel factored by one
// CTA alone (SOLO) a CTA barrier -- bar.sync orders the CTA's shared-memory
// accesses, those made through its own shared::cluster window included,
// without the cluster-scope release and acquire.
template <bool SOLO>
PFB_D void group_sync()
{
    if constexpr (SOLO) __syncthreads();
    else cluster_sync();
}

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

// ----------------------------------------------------------------- panel

// A CTA's best candidate as pushed to every CTA of the cluster: the value
// (whose modulus is the key) and its column, in one 16- or 32-byte store.
template <typename T>
struct alignas(16) PivHdr {
    T val;
    int col;
};

template <typename T, int NB>
struct PanelSmem {
    using Real = typename RealOf<T>::type;
    static constexpr int NT = kTT;
    static constexpr int NW = NT / 32;
    T lb[NB][NB + 1];                  // replicated NB x NB block of the panel columns
    alignas(16) T stage[2][NB];        // this CTA's best trailing column, panel rows 0..NB-1
    T k1col[2][NB];                    // the entries a trailing pivot column takes in the interchange
    PivHdr<T> hdr[2][kClusterMax];     // per-CTA best candidate, pushed by every CTA of the cluster
    T wval[NW];                        // per-warp best candidate
    unsigned long long wkey[NW];       // its key as bits
    int wcol[NW];
    T pivval[NB / 2];                  // this panel's pivots and pivot columns
    int pivcol[NB / 2];
};

template <typename T> PFB_D void put(uint32_t a, T v) { st_remote(a, v); }

PFB_D void put_hdr(uint32_t a, double v, int col)
{
    const long long b = __double_as_longlong(v);
    asm volatile("st.shared::cluster.v4.b32 [%0], {%1, %2, %3, %3};"
                 ::"r"(a), "r"((int)(b & 0xffffffffLL)), "r"((int)(b >> 32)), "r"(col) : "memory");
}
PFB_D void put_hdr(uint32_t a, c128 v, int col)
{
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.re), "d"(v.im) : "memory");
    asm volatile("st.shared::cluster.s32 [%0], %1;" ::"r"(a + 16), "r"(col) : "memory");
}

// The first maximum of (key, column) over a warp: the largest key (compared
// as the bits of a non-negative double, high word then low word) and, among
// equal keys, the smallest column.  Three warp reductions.
PFB_D void warp_argmax(unsigned long long kb, int col, unsigned long long &wkb, int &wcol)
{
    const unsigned hi = (unsigned)(kb >> 32), lo = (unsigned)kb;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const unsigned mc = __reduce_min_sync(0xffffffffu, (hi == mhi && lo == mlo) ? (unsigned)col : 0xffffffffu);
    wkb = ((unsigned long long)mhi << 32) | mlo;
    wcol = (int)mc;
}
PFB_D unsigned long long key_bits(double k) { return (unsigned long long)__double_as_longlong(k); }
PFB_D void store_pair(double *p, double a, double b) { *reinterpret_cast<double2 *>(p) = make_double2(a, b); }
PFB_D void store_pair(c128 *p, c128 a, c128 b) { p[0] = a; p[1] = b; }

// s + sum over the window's Gauss-vector pairs (window pair index P >= fin0,
// pair u = P - fin0) of  c_u[u] * Rw[2P+1] - c_w[u] * Rw[2P]  with
// c_u = lb[2u][col], c_w = lb[2u+1][col].  Four partial sums shorten the
// dependency chain; chunks of 8 pairs with a compiler barrier between them keep
// the coefficient loads from all being hoisted into registers at once.
template <typename T, int NB, int LBW = NB>
PFB_D T lazy_row(T s, const T (&Rw)[NB], const T (*lb)[LBW + 1], int col, int fin0)
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

// The same lazy update for a panel column c (its entries live in lb): row r
// gains sum_{u<t} lb[2u][r] lb[2u+1][c] - lb[2u+1][r] lb[2u][c], in four
// partial sums.
template <typename T, int NB>
PFB_D T lazy_panel(const T (*lb)[NB + 1], T s, int r, int c, int t)
{
    T s2 = zero<T>(), s3 = zero<T>(), s4 = zero<T>();
    int u = 0;
#pragma unroll 4
    for (; u + 1 < t; u += 2) {
        s = fma_(lb[2 * u][r], lb[2 * u + 1][c], s);
        s2 = fms_(lb[2 * u + 1][r], lb[2 * u][c], s2);
        s3 = fma_(lb[2 * u + 2][r], lb[2 * u + 3][c], s3);
        s4 = fms_(lb[2 * u + 3][r], lb[2 * u + 2][c], s4);
    }
    if (u < t) {
        s = fma_(lb[2 * u][r], lb[2 * u + 1][c], s);
        s2 = fms_(lb[2 * u + 1][r], lb[2 * u][c], s2);
    }
    return (s + s2) + (s3 + s4);
}

// Window row p (2 <= p < NB, uniform across the CTA) by a chain of selects,
// so every register index stays static.
template <typename T, int NB>
PFB_D T window_row(const T (&Rw)[NB], int p)
{
    T v = Rw[1];
#pragma unroll
    for (int i = 2; i < NB; i++) v = (i == p) ? Rw[i] : v;
    return v;
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

// Steps (2)-(4) of a pivot step, shared by both panel forms: this thread's
// best candidate (key bits kb, column col, value val; `mine`: one of this
// thread's trailing columns), the warp's best, the CTA's best -- whose header
// goes to every CTA of the cluster, and which, if it is a trailing column, its
// owner stages (stage()) -- the save of column k+1 for a trailing pivot's
// owner, the group barrier, and the pivot: its value a, column j and the CTA
// gs holding it.  Returns false for a zero pivot.
template <typename T, int NB, bool SOLO, typename Stage>
PFB_D bool pick_pivot(PanelSmem<T, NB> &sm, int t, int CL, uint32_t rank, bool has_panel, unsigned long long kb,
                      int col, T val, bool mine, Stage &&stage, T &a, int &j, int &gs)
{
    constexpr int NW = PanelSmem<T, NB>::NW;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int par = t & 1;
    unsigned long long wk;
    int wc;
    warp_argmax(kb, col, wk, wc);
    if (wc != INT_MAX && col == wc) sm.wval[warp] = val;
    if (lane == 0) { sm.wkey[warp] = wk; sm.wcol[warp] = wc; }
    __syncthreads();

    // (3) the CTA's best candidate: its header goes to every CTA of the
    // cluster, and if it is a trailing column its owner stages the column
    // (the same warp reductions over the NW warp results, lane w reading warp w's)
    const unsigned long long wkl = lane < NW ? sm.wkey[lane] : 0ull;
    const int wcl = lane < NW ? sm.wcol[lane] : INT_MAX;
    unsigned long long ck;
    int cc;
    warp_argmax(wkl, wcl, ck, cc);
    int cw = __ffs(__ballot_sync(0xffffffffu, lane < NW && wcl == cc && wkl == ck)) - 1;
    cw = cw < 0 ? 0 : cw;
    // (a CTA without candidates sends key 0 and column INT_MAX)
    if (tid < CL)
        put_hdr(map_rank(smem_u32(&sm.hdr[par][rank]), tid), cc == INT_MAX ? zero<T>() : sm.wval[cw], cc);
    if (mine && col == cc) stage();
    // if the pivot column is a trailing one, its owner fills its window
    // from column k+1 of the panel rows above k+1 and the negated row k+1
    // right of it: saved here, so that (5) can overwrite them in lb
    // without a barrier between the owner's reads and those writes
    if (has_panel) {
        const int x = tid;
        sm.k1col[par][x] = (x <= 2 * t) ? sm.lb[x][2 * t + 1]
                                        : ((x > 2 * t + 1) ? neg(sm.lb[2 * t + 1][x]) : zero<T>());
    }
    group_sync<SOLO>();

    // (4) the pivot: the first maximum over the CL <= 16 headers, lane s of
    // every warp reading header s
    T hv = zero<T>();
    int hc = INT_MAX;
    if (lane < CL) { hv = sm.hdr[par][lane].val; hc = sm.hdr[par][lane].col; }
    unsigned long long hk;
    warp_argmax(lane < CL ? key_bits(pkey(hv)) : 0ull, hc, hk, j);
    gs = __ffs(__ballot_sync(0xffffffffu, lane < CL && hc == j)) - 1;
    a = shfl(hv, gs);
    return !(is_zero(a) || j == INT_MAX);
}

// The panel-column part of the interchange k+1 <-> j (k = k0 + 2t, jl = j - k0):
// panel thread x reads the lb entries it will move (read_*), then writes them
// back permuted (write).  Thread x touches only row x and column x of lb.
template <typename T>
struct LbSwap {
    T tI = zero<T>(), tJ = zero<T>(), tRi = zero<T>(), tRj = zero<T>();

    // j is a panel column
    template <int NB>
    PFB_D void read_in_panel(const PanelSmem<T, NB> &sm, int t, int jl)
    {
        const int x = threadIdx.x;
        if (x <= 2 * t) { tI = sm.lb[x][2 * t + 1]; tJ = sm.lb[x][jl]; }
        if (x > 2 * t + 1 && x < jl) { tJ = sm.lb[x][jl]; tRi = sm.lb[2 * t + 1][x]; }
        if (x == jl) tRi = sm.lb[2 * t + 1][jl];
        if (x > jl) { tRi = sm.lb[2 * t + 1][x]; tRj = sm.lb[jl][x]; }
    }
    // j is a trailing column: its panel entries come from the stage of CTA gs
    template <int NB>
    PFB_D void read_trailing(PanelSmem<T, NB> &sm, int t, int gs)
    {
        tJ = ld_remote(map_rank(smem_u32(&sm.stage[t & 1][threadIdx.x]), (uint32_t)gs), (T *)nullptr);
    }
    template <int NB>
    PFB_D void write(PanelSmem<T, NB> &sm, int t, int jl, bool trail_win) const
    {
        const int x = threadIdx.x;
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
};

// This panel's pivots (t <= NB/2 <= 32 of them): lane s of warp 0 of rank 0
// records pivot column s and takes pivot s, then one warp tree sums the logs
// and multiplies the phases into the leader's running (la, pre + i pim).
template <typename T, int NB>
PFB_D void panel_log_pivots(const PanelSmem<T, NB> &sm, int t, int k0, uint32_t rank, bool leader,
                            int32_t *__restrict__ piv, double &la, double &pre, double &pim)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (rank != 0 || warp != 0) return;
    double lg = 0.0, ar = 1.0, ai = 0.0;
    if (lane < t) {
        const T a = sm.pivval[lane];
        piv[k0 / 2 + lane] = sm.pivcol[lane];
        const double m = (double)mag(a);
        lg = log(m);
        if constexpr (IsComplex<T>::value) { ar = a.re / m; ai = a.im / m; }
        else { ar = a < 0 ? -1.0 : 1.0; }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        lg += shfl_xor(lg, off);
        const double br = shfl_xor(ar, off), bi = shfl_xor(ai, off);
        const double nr = ar * br - ai * bi, ni = ar * bi + ai * br;
        ar = nr;
        ai = ni;
    }
    if (leader) {
        la += lg;
        const double nr = pre * ar - pim * ai, ni = pre * ai + pim * ar;
        pre = nr;
        pim = ni;
    }
}

// The factored NB x NB panel block (strict upper part) back to W, by rank 0.
template <typename T, int NB>
PFB_D void panel_store_block(const PanelSmem<T, NB> &sm, T *__restrict__ W, int n, int k0, uint32_t rank, int pc)
{
    const int tid = threadIdx.x;
    if (tid < NB && rank == 0 && pc < n)
        for (int r = 0; r < NB && r < tid; r++) W[(int64_t)(k0 + r) * n + pc] = sm.lb[r][tid];
}

PFB_D void panel_save_state(MatState *__restrict__ st, bool leader, double la, double pre, double pim, int parity)
{
    if (!leader) return;
    // keep the phase on the unit circle across panels
    const double m = sqrt(pre * pre + pim * pim);
    st->log_abs = la;
    st->ph_re = pre / m;
    st->ph_im = pim / m;
    st->parity = parity;
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
// interchanged column straight from the winning CTA's stage.  SOLO: launched
// as clusters of one CTA (the ragged kernel), the barrier is bar.sync.
template <typename T, int NB, int CPT, bool SOLO = false>
PFB_D void panel_body(PanelSmem<T, NB> &sm, T *__restrict__ W, int n, int k0, MatState *__restrict__ st,
                      int32_t *__restrict__ piv)
{
    const int tid = threadIdx.x;
    const bool has_panel = tid < NB;
    const uint32_t rank = cluster_rank();
    const int CL = (int)cluster_size();

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
    group_sync<SOLO>();

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
            const T s = lazy_panel<T, NB>(sm.lb, sm.lb[2 * t][tid], 2 * t, tid, t);
            sm.lb[2 * t][tid] = s;
            pv = s;
        }

        // (2) this thread's best candidate (its panel column first: the
        // smaller index), then the warp's.  A thread without candidates has
        // key 0 and column INT_MAX, so it loses every tie.
        unsigned long long kb = 0;
        int col = INT_MAX;
        int qsel = -1;
        T val = zero<T>();
        if (pcand) { kb = key_bits(pkey(pv)); col = pc; val = pv; }
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            if (cq[q] < n) {
                const unsigned long long kq = key_bits(pkey(Rw[q][0]));
                if (kq > kb || col == INT_MAX) { kb = kq; col = cq[q]; qsel = q; val = Rw[q][0]; }
            }
        }
        // the owner of the CTA's best trailing column stages its NB panel entries
        auto stage = [&]() {
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
        };
        T a;
        int j, gs;
        if (!pick_pivot<T, NB, SOLO>(sm, t, CL, rank, has_panel, kb, col, val, qsel >= 0, stage, a, j, gs)) {
            dead = true;
            break;
        }

        // (5) interchange k+1 <-> j on the upper triangle.  The trailing rows'
        // entries come from global memory; their loads are issued here and
        // consumed after the barriers below, so their latency overlaps them.
        T gl[CPT];
        bool gneg[CPT], guse[CPT];
        // an interchange inside the panel: window position qswap takes the old
        // row k+1 (r1s) in the rotation at the end of the step
        T r1s[CPT];
        int qswap = -1;
#pragma unroll
        for (int q = 0; q < CPT; q++) { gl[q] = zero<T>(); gneg[q] = false; guse[q] = false; r1s[q] = zero<T>(); }
        if (j != k + 1) {
            const int jl = j - k0;
            const bool trail_win = j >= k1;
            LbSwap<T> lbx;
            if (!trail_win) {
                // rows k+1 (position 1) and j (position jl - 2t) of every
                // trailing column: row j moves up now, row k+1 down in (7)
                qswap = jl - 2 * t;
#pragma unroll
                for (int q = 0; q < CPT; q++) {
                    r1s[q] = Rw[q][1];
                    Rw[q][1] = window_row<T, NB>(Rw[q], qswap);
                }
                if (has_panel) lbx.read_in_panel(sm, t, jl);
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
                            else Rw[q][p] = sm.k1col[par][r];
                        }
                    } else if (c < n) {
                        // the old row k+1 entry goes to this slot in (6), after the
                        // load has returned: a store queued behind a load of the
                        // same address would hold this thread here
                        const T *pp = (c < j) ? &W[(int64_t)c * n + j] : &W[(int64_t)j * n + c];
                        gl[q] = ldcg(pp);
                        gneg[q] = c < j;
                        guse[q] = true;
                    }
                }
                if (has_panel) lbx.read_trailing(sm, t, gs);
            }
            // no barrier here: every lb entry below is read above by the thread
            // that writes it (panel thread x reads and writes only lb[x][.] and
            // lb[.][x]), and the trailing owner of column j read k1col instead
            if (has_panel) lbx.write(sm, t, jl, trail_win);
            __syncthreads();
            parity ^= 1;
        }

        // (6) lazy update of row k+1, then u = row_k / a, w = -row_{k+1}
        const T ia = recip(a);
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            // the lazy sum first, the interchanged entry (a global load in
            // flight) last: its latency hides behind the sum
            T s1 = lazy_row<T, NB>(guse[q] ? zero<T>() : Rw[q][1], Rw[q], sm.lb, 2 * t + 1, fin0);
            if (guse[q]) {
                s1 = s1 + (gneg[q] ? neg(gl[q]) : gl[q]);
                const int c = cq[q];
                T *pp = (c < j) ? &W[(int64_t)c * n + j] : &W[(int64_t)j * n + c];
                stcg(pp, gneg[q] ? neg(Rw[q][1]) : Rw[q][1]);
            }
            Rw[q][1] = neg(s1);
            Rw[q][0] = Rw[q][0] * ia;
        }
        if (has_panel && tid > 2 * t + 1 && pc < n) {
            const T s = lazy_panel<T, NB>(sm.lb, sm.lb[2 * t + 1][tid], 2 * t + 1, tid, t);
            sm.lb[2 * t + 1][tid] = neg(s);
            sm.lb[2 * t][tid] = sm.lb[2 * t][tid] * ia;
        }
        if (tid == 0) {
            sm.pivval[t] = a;
            sm.pivcol[t] = j;
        }

        // (7) rotate the window: the finished pair goes to the end, and the old
        // row k+1 lands where row j was
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const T r0 = Rw[q][0], r1 = Rw[q][1];
#pragma unroll
            for (int p = 0; p < NB - 2; p++) Rw[q][p] = (p + 2 == qswap) ? r1s[q] : Rw[q][p + 2];
            Rw[q][NB - 2] = r0;
            Rw[q][NB - 1] = r1;
        }
        __syncthreads();
    }

    if (dead) {
        if (leader) st->dead = 1;
        group_sync<SOLO>();
        return;
    }
    panel_log_pivots(sm, t, k0, rank, leader, piv, la, pre, pim);

    // ---- write the factored panel rows back (t steps done: window position p
    // holds panel row 2t+p for p < NB-2t, else row p-(NB-2t))
#pragma unroll
    for (int q = 0; q < CPT; q++)
#pragma unroll
        for (int p = 0; p < NB; p++) {
            const int r = (p < NB - 2 * t) ? 2 * t + p : p - (NB - 2 * t);
            if (cq[q] < n && k0 + r < n) W[(int64_t)(k0 + r) * n + cq[q]] = Rw[q][p];
        }
    panel_store_block(sm, W, n, k0, rank, pc);
    panel_save_state(st, leader, la, pre, pim, parity);
    group_sync<SOLO>();
}


// ------------------------------------------- panel with half a window in smem

// The shared memory of panel_body_hs: PanelSmem plus rows NB/2 .. NB-1 of every
// trailing column's window, one column per thread (sw[r][thread]: the threads
// of a warp touch consecutive words).
template <typename T, int NB>
struct PanelSmemHS {
    PanelSmem<T, NB> base;
    alignas(16) T sw[NB / 2][kTT];
};

// The lazy sum of panel_body_hs's second phase: s + the Gauss-vector pairs
// u < NB/4 (registers, window position p = panel row p) and NB/4 <= u < t
// (sw), each  lb[2u][col] * w_u - lb[2u+1][col] * u_u  at this thread's column.
// The pairs go into the same four partial sums, in the same order, as in
// lazy_row over panel_body's window (pair u sits at window pair index
// P = u + NB/2 - t there, and P odd feeds the sums that start from s), so both
// panel forms round identically.
template <typename T, int NB>
PFB_D T lazy_mixed(T s, const T (&Rw)[NB / 2], const T (*sw)[kTT], const T (*lb)[NB + 1], int col, int t)
{
    constexpr int NR = NB / 2;
    const int x = threadIdx.x;
    const bool todd = t & 1;
    // e: pairs with u even, o: u odd; the (u + t)-odd pair of sums starts from s
    T e1 = todd ? s : zero<T>(), e2 = zero<T>();
    T o1 = todd ? zero<T>() : s, o2 = zero<T>();
#pragma unroll
    for (int u = 0; u < NR / 2; u += 2) {
        e1 = fma_(lb[2 * u][col], Rw[2 * u + 1], e1);
        e2 = fms_(lb[2 * u + 1][col], Rw[2 * u], e2);
        o1 = fma_(lb[2 * u + 2][col], Rw[2 * u + 3], o1);
        o2 = fms_(lb[2 * u + 3][col], Rw[2 * u + 2], o2);
    }
    int u = NR / 2;   // even
#pragma unroll 1
    for (; u + 1 < t; u += 2) {
        e1 = fma_(lb[2 * u][col], sw[2 * u + 1 - NR][x], e1);
        e2 = fms_(lb[2 * u + 1][col], sw[2 * u - NR][x], e2);
        o1 = fma_(lb[2 * u + 2][col], sw[2 * u + 3 - NR][x], o1);
        o2 = fms_(lb[2 * u + 3][col], sw[2 * u + 2 - NR][x], o2);
    }
    if (u < t) {
        e1 = fma_(lb[2 * u][col], sw[2 * u + 1 - NR][x], e1);
        e2 = fms_(lb[2 * u + 1][col], sw[2 * u - NR][x], e2);
    }
    return todd ? (e1 + e2) + (o1 + o2) : (o1 + o2) + (e1 + e2);
}

// panel_body for one trailing column per thread, with rows 0 .. NB/2-1 of the
// column's window in registers and rows NB/2 .. NB-1 in shared memory (sw):
// half the registers of panel_body's window, so two CTAs share an SM and twice
// as many panel clusters run at once (the pivot steps are latency-bound, so two
// CTAs interleave on one SM at little cost to either).  Same algorithm, same
// pivots and the same rounding as panel_body.
//   phase 1 (t < NB/4): the pivot rows come from the registers, which rotate as
//     in panel_body (position p = row 2t+p for p < NB/2-2t, else row
//     p-(NB/2-2t)); sw holds raw rows, and an interchange with a row there
//     swaps it with row k+1 at once;
//   phase 2: the registers hold the Gauss vectors of pairs 0 .. NB/4-1 in
//     natural order (position p = row p); rows k, k+1 and the later pairs are
//     read and written in sw in place, nothing rotates.
template <typename T, int NB, bool SOLO = false>
PFB_D void panel_body_hs(PanelSmemHS<T, NB> &smh, T *__restrict__ W, int n, int k0, MatState *__restrict__ st,
                         int32_t *__restrict__ piv)
{
    constexpr int NR = NB / 2;   // window rows in registers
    static_assert(NR % 4 == 0, "pairs of pairs in the register half");
    PanelSmem<T, NB> &sm = smh.base;
    T (*sw)[kTT] = smh.sw;
    const int tid = threadIdx.x;
    const bool has_panel = tid < NB;
    const uint32_t rank = cluster_rank();
    const int CL = (int)cluster_size();

    if (st->dead) return;   // same value for the whole cluster

    const int k1 = k0 + NB;
    const int pc = k0 + tid;                      // panel column of this thread (if has_panel)
    const int cq = k1 + (int)rank * kTT + tid;    // trailing column of this thread
    const bool own = cq < n;

    T Rw[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) Rw[r] = (own && k0 + r < n) ? W[(int64_t)(k0 + r) * n + cq] : zero<T>();
#pragma unroll 4
    for (int r = NR; r < NB; r++) sw[r - NR][tid] = (own && k0 + r < n) ? W[(int64_t)(k0 + r) * n + cq] : zero<T>();
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
    group_sync<SOLO>();

    // a panel-column candidate (the smaller index) first, then the trailing one
    auto panel_candidate = [&](int t, unsigned long long &kb, int &col, T &val) {
        if (has_panel && tid > 2 * t && pc < n) {
            const T s = lazy_panel<T, NB>(sm.lb, sm.lb[2 * t][tid], 2 * t, tid, t);
            sm.lb[2 * t][tid] = s;
            kb = key_bits(pkey(s));
            col = pc;
            val = s;
        }
    };
    auto panel_finish = [&](int t, T a, int j, T ia) {
        if (has_panel && tid > 2 * t + 1 && pc < n) {
            const T s = lazy_panel<T, NB>(sm.lb, sm.lb[2 * t + 1][tid], 2 * t + 1, tid, t);
            sm.lb[2 * t + 1][tid] = neg(s);
            sm.lb[2 * t][tid] = sm.lb[2 * t][tid] * ia;
        }
        if (tid == 0) {
            sm.pivval[t] = a;
            sm.pivcol[t] = j;
        }
    };

    int t = 0;
    // ---- phase 1
#pragma unroll 1
    for (; t < nsteps && t < NR / 2; t++) {
        const int k = k0 + 2 * t;
        const int par = t & 1;
        const int fin0 = NR / 2 - t;

        Rw[0] = lazy_row<T, NR, NB>(Rw[0], Rw, sm.lb, 2 * t, fin0);
        unsigned long long kb = 0;
        int col = INT_MAX;
        T val = zero<T>();
        panel_candidate(t, kb, col, val);
        bool mine = false;
        if (own) {
            const unsigned long long kq = key_bits(pkey(Rw[0]));
            if (kq > kb || col == INT_MAX) { kb = kq; col = cq; mine = true; val = Rw[0]; }
        }
        auto stage = [&]() {
#pragma unroll
            for (int P = 0; P < NR / 2; P++) {
                const int r = (2 * P < NR - 2 * t) ? 2 * t + 2 * P : 2 * P - (NR - 2 * t);
                store_pair(&sm.stage[par][r], Rw[2 * P], Rw[2 * P + 1]);
            }
#pragma unroll 4
            for (int r = NR; r < NB; r += 2) store_pair(&sm.stage[par][r], sw[r - NR][tid], sw[r + 1 - NR][tid]);
        };
        T a;
        int j, gs;
        if (!pick_pivot<T, NB, SOLO>(sm, t, CL, rank, has_panel, kb, col, val, mine, stage, a, j, gs)) {
            dead = true;
            break;
        }

        T gl = zero<T>(), r1s = zero<T>();
        bool gneg = false, guse = false;
        int qswap = -1;
        if (j != k + 1) {
            const int jl = j - k0;
            const bool trail_win = j >= k1;
            LbSwap<T> lbx;
            if (!trail_win) {
                if (jl < NR) {
                    // row j at register position jl - 2t moves up now, row k+1 down in the rotation
                    qswap = jl - 2 * t;
                    r1s = Rw[1];
                    Rw[1] = window_row<T, NR>(Rw, qswap);
                } else {
                    const T x = sw[jl - NR][tid];
                    sw[jl - NR][tid] = Rw[1];
                    Rw[1] = x;
                }
                if (has_panel) lbx.read_in_panel(sm, t, jl);
            } else {
                if (cq == j) {
                    // the new column j: rows < k+1 from column k+1, (k+1, j)
                    // negated, rows > k+1 (all of sw) from row k+1 negated
#pragma unroll
                    for (int p = 0; p < NR; p++) {
                        const int r = (p < NR - 2 * t) ? 2 * t + p : p - (NR - 2 * t);
                        if (p == 1) Rw[1] = neg(Rw[1]);
                        else Rw[p] = sm.k1col[par][r];
                    }
#pragma unroll 4
                    for (int r = NR; r < NB; r++) sw[r - NR][tid] = sm.k1col[par][r];
                } else if (own) {
                    const T *pp = (cq < j) ? &W[(int64_t)cq * n + j] : &W[(int64_t)j * n + cq];
                    gl = ldcg(pp);
                    gneg = cq < j;
                    guse = true;
                }
                if (has_panel) lbx.read_trailing(sm, t, gs);
            }
            if (has_panel) lbx.write(sm, t, jl, trail_win);
            __syncthreads();
            parity ^= 1;
        }

        const T ia = recip(a);
        T s1 = lazy_row<T, NR, NB>(guse ? zero<T>() : Rw[1], Rw, sm.lb, 2 * t + 1, fin0);
        if (guse) {
            s1 = s1 + (gneg ? neg(gl) : gl);
            T *pp = (cq < j) ? &W[(int64_t)cq * n + j] : &W[(int64_t)j * n + cq];
            stcg(pp, gneg ? neg(Rw[1]) : Rw[1]);
        }
        Rw[1] = neg(s1);
        Rw[0] = Rw[0] * ia;
        panel_finish(t, a, j, ia);

        // rotate the register window; the old row k+1 lands where row j was
        {
            const T r0 = Rw[0], r1 = Rw[1];
#pragma unroll
            for (int p = 0; p < NR - 2; p++) Rw[p] = (p + 2 == qswap) ? r1s : Rw[p + 2];
            Rw[NR - 2] = r0;
            Rw[NR - 1] = r1;
        }
        __syncthreads();
    }

    // ---- phase 2
#pragma unroll 1
    for (; !dead && t < nsteps; t++) {
        const int k = k0 + 2 * t;
        const int par = t & 1;
        const int s0 = 2 * t - NR, s1 = s0 + 1;   // sw rows of k and k+1

        const T rk = lazy_mixed<T, NB>(sw[s0][tid], Rw, sw, sm.lb, 2 * t, t);
        sw[s0][tid] = rk;
        unsigned long long kb = 0;
        int col = INT_MAX;
        T val = zero<T>();
        panel_candidate(t, kb, col, val);
        bool mine = false;
        if (own) {
            const unsigned long long kq = key_bits(pkey(rk));
            if (kq > kb || col == INT_MAX) { kb = kq; col = cq; mine = true; val = rk; }
        }
        auto stage = [&]() {
#pragma unroll
            for (int P = 0; P < NR / 2; P++) store_pair(&sm.stage[par][2 * P], Rw[2 * P], Rw[2 * P + 1]);
#pragma unroll 4
            for (int r = NR; r < NB; r += 2) store_pair(&sm.stage[par][r], sw[r - NR][tid], sw[r + 1 - NR][tid]);
        };
        T a;
        int j, gs;
        if (!pick_pivot<T, NB, SOLO>(sm, t, CL, rank, has_panel, kb, col, val, mine, stage, a, j, gs)) {
            dead = true;
            break;
        }

        T gl = zero<T>();
        bool gneg = false, guse = false;
        if (j != k + 1) {
            const int jl = j - k0;
            const bool trail_win = j >= k1;
            LbSwap<T> lbx;
            if (!trail_win) {
                const T x = sw[jl - NR][tid];
                sw[jl - NR][tid] = sw[s1][tid];
                sw[s1][tid] = x;
                if (has_panel) lbx.read_in_panel(sm, t, jl);
            } else {
                if (cq == j) {
#pragma unroll
                    for (int p = 0; p < NR; p++) Rw[p] = sm.k1col[par][p];
#pragma unroll 4
                    for (int r = NR; r < NB; r++)
                        sw[r - NR][tid] = (r == 2 * t + 1) ? neg(sw[r - NR][tid]) : sm.k1col[par][r];
                } else if (own) {
                    const T *pp = (cq < j) ? &W[(int64_t)cq * n + j] : &W[(int64_t)j * n + cq];
                    gl = ldcg(pp);
                    gneg = cq < j;
                    guse = true;
                }
                if (has_panel) lbx.read_trailing(sm, t, gs);
            }
            if (has_panel) lbx.write(sm, t, jl, trail_win);
            __syncthreads();
            parity ^= 1;
        }

        const T ia = recip(a);
        const T raw1 = sw[s1][tid];
        T v1 = lazy_mixed<T, NB>(guse ? zero<T>() : raw1, Rw, sw, sm.lb, 2 * t + 1, t);
        if (guse) {
            v1 = v1 + (gneg ? neg(gl) : gl);
            T *pp = (cq < j) ? &W[(int64_t)cq * n + j] : &W[(int64_t)j * n + cq];
            stcg(pp, gneg ? neg(raw1) : raw1);
        }
        sw[s1][tid] = neg(v1);
        sw[s0][tid] = sw[s0][tid] * ia;
        panel_finish(t, a, j, ia);
        __syncthreads();
    }

    if (dead) {
        if (leader) st->dead = 1;
        group_sync<SOLO>();
        return;
    }
    panel_log_pivots(sm, t, k0, rank, leader, piv, la, pre, pim);

    // ---- write the factored panel rows back: registers in the phase-1
    // arrangement if the panel ended there (t <= NB/4), else in natural order
    if (own) {
        const int tr = t < NR / 2 ? t : NR / 2;
#pragma unroll
        for (int p = 0; p < NR; p++) {
            const int r = (p < NR - 2 * tr) ? 2 * tr + p : p - (NR - 2 * tr);
            if (k0 + r < n) W[(int64_t)(k0 + r) * n + cq] = Rw[p];
        }
#pragma unroll 4
        for (int r = NR; r < NB; r++)
            if (k0 + r < n) W[(int64_t)(k0 + r) * n + cq] = sw[r - NR][tid];
    }
    panel_store_block(sm, W, n, k0, rank, pc);
    panel_save_state(st, leader, la, pre, pim, parity);
    group_sync<SOLO>();
}

}  // namespace pfb
