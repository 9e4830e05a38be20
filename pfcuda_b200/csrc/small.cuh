// small.cuh -- launcher of the small-matrix kernel (n <= 32), see small.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pfb {
// slog = false: out_val[b] = Pf (dtype).  slog = true: out_log[b] = log|Pf|,
// out_sign[b] = sign / phase (dtype).
int launch_small(int dtype, bool slog, const void *A, int64_t batch, int n, int layout,
                 void *out_val, double *out_log, void *out_sign, cudaStream_t stream);
}  // namespace pfb
