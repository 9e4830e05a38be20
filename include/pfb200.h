/*
 * pfb200.h -- C ABI of the B200 Pfaffian engine (libpfb200.so).
 *
 * Plain C types only: device pointers, sizes, enums and a cudaStream_t passed as
 * void*.  Every entry point
 *   - enqueues its work on `stream` and returns without synchronising the host,
 *   - allocates no device memory: scratch memory is the caller's `workspace`,
 *     whose size the matching *_workspace_bytes function gives (the one
 *     exception, pfb_slog_pfaffian_noalloc, says how it differs),
 *   - never throws and never writes its input; errors come back as a pfb_status,
 *   - is re-entrant, so several streams or threads may call it at once: the only
 *     state kept between calls is read-only after its first use (device
 *     properties, the split kernel's tensor-map entry point) or private to the
 *     calling host thread (the second stream of pfb_slog_stream_ranges).
 *
 * Matrices are batches of `batch` contiguous n x n arrays.  `layout` says how one
 * matrix is stored: PFB_ROW_MAJOR (C order, torch/NumPy default) or PFB_COL_MAJOR
 * (how XLA hands a matrix to the reference's handlers, which request
 * input_layouts=[(1, 0)] at pfcuda/cuda_api.py:50,72 and index CM(A,n,r,c) =
 * A[r + c*n], include/pfaffian_utils.cuh:10).  The inputs are taken to be
 * skew-symmetric; the Pfaffian of the matrix in the stated layout is returned.
 *
 * Complex values are interleaved (re, im) pairs of float (C64) or double (C128).
 */
#ifndef PFB200_H
#define PFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PFB_F32 = 0,   /* float            */
    PFB_F64 = 1,   /* double           */
    PFB_C64 = 2,   /* complex float    */
    PFB_C128 = 3   /* complex double   */
} pfb_dtype;

typedef enum {
    PFB_ROW_MAJOR = 0,
    PFB_COL_MAJOR = 1
} pfb_layout;

/* Arithmetic of the trailing skew rank-2k update of the blocked factorisation.
 * The panel (pivot search, interchanges, Gauss vectors, log|Pf| and sign) is
 * always FP64 (complex128 for complex input). */
typedef enum {
    PFB_MODE_FP64 = 0,   /* FP64 / complex128 update                                */
    PFB_MODE_SPLIT = 1   /* error-free int8 slices on the tcgen05 tensor cores with
                            exact int32 accumulation, recombined in FP64             */
} pfb_mode;
/* For PFB_MODE_SPLIT, bits 8..11 of `mode` may give the number of 7-bit int8
 * digits per operand (1..7; 0 selects the default, 7).  Fewer digits trade
 * accuracy for speed: S digits keep the update to about K * 2^(-7S) relative. */
#define PFB_SPLIT_DIGITS(s) ((s) << 8)
/* Test only, PFB_MODE_SPLIT: every bounded device-side wait of the split
 * update's pipeline for the first matrix of the call gives up without polling,
 * exactly as a wait that ran out of its bound would.  That matrix's result is
 * log = NaN, sign = 0 (the update kernel lets its copies and MMAs in flight land
 * and frees its tensor memory before it returns); the other matrices of the
 * call are unaffected and the device stays usable. */
#define PFB_SPLIT_TEST_TIMEOUT (1 << 12)

typedef enum {
    PFB_OK = 0,
    PFB_ERR_INVALID = 1,     /* null pointer, bad enum, negative batch        */
    PFB_ERR_SIZE = 2,        /* matrix order outside the entry point's range  */
    PFB_ERR_WORKSPACE = 3,   /* workspace missing, too small or misaligned    */
    PFB_ERR_CUDA = 4,        /* a CUDA runtime call failed                    */
    PFB_ERR_UNSUPPORTED = 5, /* combination not built (e.g. no sm_100a device) */
    PFB_ERR_TIMEOUT = 6      /* a bounded device-side wait gave up            */
} pfb_status;

/* Text for a status code (static storage). */
const char *pfb_status_string(int status);

/* Last CUDA error seen by the calling thread's most recent failing call. */
int pfb_last_cuda_error(void);

/*
 * Pf(A) for n <= 32, one value per matrix, in the input dtype.
 *
 * Replaces the XLA handlers pfaffian_f32 / _f64 / _c64 / _c128
 * (bindings/jax_bindings.cu:82-112, symbols :152-183), which launch the
 * reference kernel pf_sm_calc once per matrix (src/pfaffian_sm.cu:101-105).
 * Here one launch covers the whole batch.  n == 0 or odd gives 0; n > 32 gives
 * PFB_ERR_SIZE (the reference throws, src/pfaffian.cu:44-45).  A zero pivot
 * gives 0.  out: `batch` values of `dtype`.  No workspace.
 */
int pfb_pfaffian(int dtype, const void *A, int64_t batch, int n, int layout,
                 void *out, void *stream);

/*
 * (log|Pf|, sign) for any even n.
 *
 * Replaces the XLA handlers slog_pfaffian_f32 / _f64 / _c64 / _c128
 * (bindings/jax_bindings.cu:19-80, symbols :115-150), which copy each matrix
 * and run the host-driven loop of src/slog_pfaffian_lg.cu:151-211.
 * log_out: `batch` doubles (pfcuda/cuda_api.py:71 declares the log as float64).
 * sign_out: `batch` values of `dtype`: +-1 for real input, a unit-modulus
 * phase for complex input, 0 when Pf = 0 (then log = -inf).  Odd n gives
 * (-inf, 0).  n <= 32 is accepted too (the Python layer refuses it as the
 * reference does, cuda_api.py:60-61).  f32 / c64 input is evaluated in FP64 /
 * complex128.
 * workspace: at least pfb_slog_workspace_bytes(dtype, batch, n, mode) bytes,
 * 256-byte aligned.
 */
int pfb_slog_pfaffian(int dtype, const void *A, int64_t batch, int n, int layout,
                      int mode, double *log_out, void *sign_out,
                      void *workspace, size_t workspace_bytes, void *stream);

size_t pfb_slog_workspace_bytes(int dtype, int64_t batch, int n, int mode);

/*
 * Optional instrumentation for pfb_slog_pfaffian_timed: caller-created CUDA
 * events (cudaEvent_t passed as void*), recorded on `stream` around each launch
 * of the panel kernel and of the trailing-update kernel(s).  Entry 2i / 2i+1 of
 * each array is the start / stop of the i-th panel (update); at most `pairs`
 * pairs are recorded per array.  The number of panels is ceil((n-1)/nb) with
 * nb = pfb_slog_panel_width(dtype, n).
 */
typedef struct {
    void **panel_events;
    void **update_events;
    int pairs;
} pfb_slog_timing;

/* pfb_slog_pfaffian with event records around its kernels (timing may be NULL). */
int pfb_slog_pfaffian_timed(int dtype, const void *A, int64_t batch, int n, int layout,
                            int mode, double *log_out, void *sign_out,
                            void *workspace, size_t workspace_bytes, void *stream,
                            const pfb_slog_timing *timing);

/*
 * Settings of the large path that do not change its results' meaning, only
 * how the work maps onto the GPU (and, for the split update, how many int8
 * digits carry each operand).  Zero fields take the tuned table's choice for
 * (dtype, n, batch): a table measured on the B200 by pfcuda_b200/tune.py and
 * compiled into the library (pfcuda_b200/tune_table.json).
 *   panel:  PFB_PANEL_REGISTERS -- each trailing column's panel rows in the
 *           registers of one thread, one CTA per SM;
 *           PFB_PANEL_HALF_SHARED -- half of those rows in shared memory, two
 *           CTAs per SM, twice as many matrices' panels at once (orders whose
 *           panel puts one trailing column per thread: up to 4160 real,
 *           2080 complex).
 *           Both forms choose the same pivots and round identically.
 *   slices: int8 digits per operand of the split update (1..7); the mode's
 *           PFB_SPLIT_DIGITS bits, when set, take precedence over the table.
 *   ranges: 1 -- one stream; 2 -- a batch of two or more waves of the widest
 *           panel clusters runs as two ranges (pfb_slog_stream_ranges).
 *   epilogue (split update, 5 to 7 digits): PFB_EPILOGUE_ROUNDTRIP -- each
 *           FP64 tile of the working matrix comes into shared memory by TMA,
 *           is updated there and goes back by TMA; PFB_EPILOGUE_REDUCE -- only
 *           the tile's increment is formed, and the L2 adds it to the working
 *           matrix (bulk reduce-add); PFB_EPILOGUE_DIRECT (real
 *           input; complex input takes the round trip) -- each tile is formed
 *           transposed, so that the lanes of a warp hold adjacent columns of
 *           C, which is then read and written straight from global memory in
 *           coalesced row segments (only the strictly upper part is
 *           written).  All three round identically: one rounding of
 *           C + increment, the increment exact.
 */
typedef enum {
    PFB_PANEL_REGISTERS = 1,
    PFB_PANEL_HALF_SHARED = 2
} pfb_panel_form;

typedef enum {
    PFB_EPILOGUE_ROUNDTRIP = 1,
    PFB_EPILOGUE_REDUCE = 2,
    PFB_EPILOGUE_DIRECT = 3
} pfb_split_epilogue;

typedef struct {
    int panel;
    int slices;
    int ranges;
    int epilogue;
} pfb_slog_config;

/* The configuration a pfb_slog_pfaffian call on these arguments uses (the
 * tuned table's choice), in *out.  Returns PFB_ERR_SIZE for orders outside the
 * large path. */
int pfb_slog_config_for(int dtype, int64_t batch, int n, int mode, pfb_slog_config *out);

/* pfb_slog_pfaffian_timed with the configuration's non-zero fields in place of
 * the table's (config may be NULL); PFB_ERR_INVALID for a field out of range or
 * a panel form the order does not have. */
int pfb_slog_pfaffian_ex(int dtype, const void *A, int64_t batch, int n, int layout,
                         int mode, double *log_out, void *sign_out,
                         void *workspace, size_t workspace_bytes, void *stream,
                         const pfb_slog_timing *timing, const pfb_slog_config *config);

/* Panel width (pivot rows per panel) the blocked factorisation uses for this
 * dtype and order; 0 if the order is not supported. */
int pfb_slog_panel_width(int dtype, int n);

/*
 * How many matrices of order n the current device factors concurrently: the
 * number of panel thread-block clusters (one per matrix, up to 16 CTAs) that
 * can be resident at once for the widest panel of the factorisation, as the
 * CUDA occupancy calculator reports it, for the PFB_PANEL_REGISTERS form (7 on
 * a B200 for 2n = 4096; PFB_PANEL_HALF_SHARED fits about twice as many).  A
 * batch of this many matrices keeps every panel in one wave.  Returns 0 for
 * orders the large path does not take, or without a device.  No reference
 * counterpart.
 */
int pfb_slog_max_concurrent(int dtype, int n);

/* The same count for a given panel form (pfb_panel_form); 0 if the order does
 * not have that form. */
int pfb_slog_max_concurrent_form(int dtype, int n, int panel);

/*
 * How many ranges a pfb_slog_pfaffian call on `batch` matrices of order n runs
 * as (1 or 2), for the tuned table's configuration in `mode` (PFB_MODE_*).  When
 * the configuration asks for two ranges and the widest panel clusters have 9 or
 * more CTAs, a batch of three or more waves of them is split in two -- the last
 * wave's worth of matrices on a second stream -- and a batch of two waves into
 * halves; the second stream forks from and joins `stream` through events, so
 * one range's trailing updates fill the SMs the other's panel waves leave idle.  The second stream belongs to the calling host thread (one per
 * thread and device, created on its first use and destroyed when the thread
 * exits), so calls from different threads never share it; a call whose
 * thread's second stream is part of another graph capture runs as one range.
 * Each range launches its own sequence of kernels.  No reference counterpart.
 */
int pfb_slog_stream_ranges(int dtype, int64_t batch, int n, int mode);

/*
 * pfb_slog_pfaffian on a batch given as matrix pointers: A_ptrs is a DEVICE
 * array of `batch` pointers, each to one contiguous n x n matrix of `dtype` in
 * `layout` (the matrices need not be adjacent or in order).  n must be even and
 * above 32 (PFB_ERR_SIZE otherwise).  Results, workspace
 * (pfb_slog_workspace_bytes) and configuration are those of pfb_slog_pfaffian.
 * It serves ragged batches whose orders exceed PFB_RAGGED_MAX_N: one call per
 * order on the matrices of that order, wherever they lie.  No reference
 * counterpart (the reference's caller loops over matrices,
 * pfcuda/cuda_api.py:57-76).
 */
int pfb_slog_pfaffian_ptrs(int dtype, const void *const *A_ptrs, int64_t batch, int n, int layout,
                           int mode, double *log_out, void *sign_out, void *workspace,
                           size_t workspace_bytes, void *stream);

/*
 * (log|Pf|, sign) of a ragged batch in one launch: `count` matrices of even (or
 * odd) orders n[i] <= max_n <= PFB_RAGGED_MAX_N, each float32 or float64
 * (dtype[i]), each contiguous at A[i] in `layout`.  A, n and dtype are DEVICE
 * arrays.  log_out[i] and sign_out[i] are doubles (sign +-1, or 0 with
 * log = -inf when Pf = 0 or the order is odd; log = NaN for an order above
 * max_n or an unknown dtype).  Every matrix is factored in FP64.
 *
 * No counterpart call in the reference, whose caller loops over sizes and calls
 * slog_pfaffian per matrix (pfcuda/cuda_api.py:57-76, each a host-driven loop,
 * src/slog_pfaffian_lg.cu:151-211).  Nothing is allocated and the host is not
 * synchronised, so the call may be captured in a CUDA graph and replayed.
 * workspace: pfb_slog_ragged_workspace_bytes(count, max_n) bytes, 256-aligned.
 */
#define PFB_RAGGED_MAX_N 544
int pfb_slog_pfaffian_ragged(const void *const *A, const int32_t *n, const int32_t *dtype,
                             int64_t count, int max_n, int layout, double *log_out,
                             double *sign_out, void *workspace, size_t workspace_bytes,
                             void *stream);

size_t pfb_slog_ragged_workspace_bytes(int64_t count, int max_n);

/*
 * Pivot columns chosen by the last pfb_slog_pfaffian call that used this
 * workspace: n/2 int32 per matrix (the column index swapped into position k+1
 * at pivot step k, as the reference's argmax picks it).  Copies into the device
 * buffer `piv_out` on `stream`.
 */
int pfb_slog_pivots(int64_t batch, int n, const void *workspace, size_t workspace_bytes,
                    int32_t *piv_out, void *stream);

/*
 * pfb_slog_pfaffian without a caller workspace.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory (a plugin
 * given raw pointers by a framework that owns all allocations, a binding with no
 * CUDA allocator, a path where a device-synchronising cudaMalloc is not
 * acceptable).  The scratch is one array of PFB_NOALLOC_SCRATCH_BYTES inside
 * libpfb200.so, held on every GPU that loads the library until exit.
 *   - Sizes whose pfb_slog_workspace_bytes(dtype, batch, n, mode) exceeds
 *     PFB_NOALLOC_SCRATCH_BYTES return PFB_ERR_SIZE (n <= 32 needs no scratch);
 *     e.g. one float64 matrix fits up to n = 1448 (1392 in PFB_MODE_SPLIT), one
 *     complex128 matrix up to n = 1022 (980 in PFB_MODE_SPLIT).
 *   - Every call looks up the array's device address on the current device
 *     (nothing is cached, so a device reset between calls is harmless); the
 *     first call on a device also loads the library's module there, so make
 *     that first call before any stream capture.
 *   - All calls share the array: calls that overlap on the GPU race and must be
 *     serialised by the caller.
 * Nothing is allocated; arguments and results are those of pfb_slog_pfaffian.
 */
#define PFB_NOALLOC_SCRATCH_BYTES (16u << 20)
int pfb_slog_pfaffian_noalloc(int dtype, const void *A, int64_t batch, int n, int layout,
                              int mode, double *log_out, void *sign_out, void *stream);

/*
 * Reverse-mode derivative of log|Pf(A)|, fused with the forward pass.
 * Replaces the reference's differentiation rule slog_pfaffian_jvp
 * (pfcuda/cuda_api.py:92-107), which calls jnp.linalg.inv:
 *     d log Pf = (1/2) tr(A^-1 dA)   =>   d log Pf / dA = (1/2) A^-T
 * (holomorphic: no conjugation; a torch or JAX wrapper conjugates as its own
 * convention asks).  The inverse comes from the engine's own blocked skew-LTL^T
 * factors, not from a general LU.
 *   G_out[b] = ct_log[b] * (1/2) A[b]^-T, in the dtype and layout of A;
 *   ct_log: batch float64 cotangents on the device, or NULL for all ones;
 *   log_out / sign_out: the forward results, exactly as pfb_slog_pfaffian;
 *   a matrix with Pf = 0 gets an all-NaN gradient.
 * n must be even (odd orders have Pf = 0 identically: PFB_ERR_SIZE) and within
 * the large path's range.
 * workspace (256-aligned) is the call's memory budget: about 2 n^2 elements of
 * the working type per matrix (the factors and the inverse of their unit
 * triangle), pfb_slog_grad_workspace_bytes(dtype, batch, n, mode) for the whole
 * batch at once.  Any smaller workspace of at least
 * pfb_slog_grad_workspace_bytes(dtype, 1, n, mode) bytes is accepted: the batch
 * then runs in chunks of as many matrices as fit, each chunk's factors formed,
 * used and overwritten by the next chunk's.  Results do not depend on the
 * chunking (every matrix's arithmetic is its own).  The reference's rule keeps
 * no factors but calls a general inverse per matrix (cuda_api.py:84-89).
 */
int pfb_slog_pfaffian_grad(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                           const double *ct_log, void *G_out, double *log_out, void *sign_out,
                           void *workspace, size_t workspace_bytes, void *stream);

size_t pfb_slog_grad_workspace_bytes(int dtype, int64_t batch, int n, int mode);

/*
 * Host -> device upload of a batch for pfb_slog_pfaffian that moves only what
 * the large path reads: in the row-major view of each matrix (either layout),
 * the entries on and above the diagonal, as one rectangle per block of 256
 * rows (rows [r0, r0+256) x columns [r0, n)) -- about (n^2 + 256 n) / 2
 * elements per matrix instead of n^2.  Entries below the diagonal of A_dev are
 * left as they were: the large path never reads them.  Orders n <= 32 (the
 * small path, which reads whole matrices) are copied whole.  A_host: `batch`
 * contiguous n x n matrices in host memory, page-locked for the copies to be
 * asynchronous on `stream`; A_dev: a contiguous device array of the same
 * shape and dtype.  No counterpart in the reference, whose handlers receive
 * device buffers from XLA (bindings/jax_bindings.cu:19-80); its CPU path reads
 * the same triangle (src/pfaffian_cpu.cpp:33-42).
 */
int pfb_upload_upper(int dtype, const void *A_host, void *A_dev, int64_t batch, int n, void *stream);

/* Bytes pfb_upload_upper moves for such a batch (0 for invalid arguments). */
size_t pfb_upload_upper_bytes(int dtype, int64_t batch, int n);

#ifdef __cplusplus
}
#endif

#endif /* PFB200_H */
