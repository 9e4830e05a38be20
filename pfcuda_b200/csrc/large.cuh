// large.cuh -- blocked skew-LTL^T factorisation for (log|Pf|, sign) of large
// matrices, see large.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/pfb200.h"

namespace pfb {

// Per-matrix running state of the factorisation, kept in the workspace.
struct __align__(64) MatState {
    double log_abs;   // sum of log|pivot|
    double ph_re;     // product of pivot / |pivot| (imaginary part 0 for real input)
    double ph_im;
    int parity;       // number of interchanges mod 2
    int dead;         // a zero pivot was met: Pf = 0
};

size_t large_workspace_bytes(int dtype, int64_t batch, int n, int mode);

int launch_large(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                 double *log_out, void *sign_out, void *workspace, size_t workspace_bytes,
                 cudaStream_t stream, const pfb_slog_timing *timing, const pfb_slog_config *config = nullptr,
                 const void *const *A_ptrs = nullptr);
bool large_config(int dtype, int64_t batch, int n, int mode, const pfb_slog_config *over, pfb_slog_config *out);

int large_panel_width(int dtype, int n);
int large_max_concurrent(int dtype, int n, int panel);
int64_t large_second_range(int dtype, int64_t batch, int n, const pfb_slog_config &cf);

// Where the factorisation leaves its results inside a large-path workspace:
// the pivot columns (n/2 per matrix), the per-matrix state, and W, the
// FP64 / complex128 working matrices holding the Gauss vectors (row 2t = u_t,
// row 2t+1 = w_t right of column 2t+1, W[2t][2t+1] = the pivot a_t).
struct LargeView {
    int32_t *piv;
    MatState *st;
    void *W;
};
LargeView large_view(int dtype, int64_t batch, int n, int mode, void *workspace);

// Declared here, defined in grad.cu: the adjoint of log|Pf|.
size_t grad_workspace_bytes(int dtype, int64_t batch, int n, int mode);
int64_t grad_chunk(int dtype, int64_t batch, int n, int mode, size_t bytes);
int launch_grad(int dtype, const void *A, int64_t batch, int n, int layout, int mode, const double *ct, void *G,
                double *log_out, void *sign_out, void *workspace, size_t workspace_bytes, cudaStream_t stream);

size_t ragged_workspace_bytes(int64_t count, int max_n);
int launch_ragged(const void *const *A, const int32_t *n, const int32_t *dtype, int64_t count, int max_n,
                  int layout, double *log_out, double *sign_out, void *workspace, cudaStream_t s);

int large_copy_pivots(int64_t batch, int n, const void *workspace, size_t workspace_bytes,
                      int32_t *piv_out, cudaStream_t stream);

}  // namespace pfb
