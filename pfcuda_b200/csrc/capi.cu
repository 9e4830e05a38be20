// capi.cu -- the extern "C" entry points declared in include/pfb200.h.
//
// Argument checking and dispatch only; the kernels live in small.cu and
// large.cu.  Nothing here allocates device memory or synchronises the host.
#include <string.h>

#include "common.cuh"
#include "small.cuh"
#include "large.cuh"

namespace {
thread_local int g_last_cuda_error = 0;

int cuda_status(cudaError_t e) { return pfb::cuda_check(e); }

// A call that failed with PFB_ERR_CUDA recorded its error where it happened; a
// runtime error still pending (a failed attribute call, say) is recorded too.
int cuda_failed()
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) g_last_cuda_error = (int)e;
    return PFB_ERR_CUDA;
}

bool valid_dtype(int d) { return d == PFB_F32 || d == PFB_F64 || d == PFB_C64 || d == PFB_C128; }
bool valid_layout(int l) { return l == PFB_ROW_MAJOR || l == PFB_COL_MAJOR; }

size_t dtype_bytes(int d) { return d == PFB_F32 ? 4 : (d == PFB_C128 ? 16 : 8); }

constexpr int kUploadRows = 256;   // rows per rectangle of pfb_upload_upper
}  // namespace

namespace pfb {
int &last_cuda_error() { return g_last_cuda_error; }
}

extern "C" {

const char *pfb_status_string(int status)
{
    switch (status) {
    case PFB_OK: return "ok";
    case PFB_ERR_INVALID: return "invalid argument";
    case PFB_ERR_SIZE: return "matrix order outside the supported range";
    case PFB_ERR_WORKSPACE: return "workspace missing, too small or misaligned";
    case PFB_ERR_CUDA: return "CUDA runtime error";
    case PFB_ERR_UNSUPPORTED: return "unsupported combination";
    case PFB_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
    }
}

int pfb_last_cuda_error(void) { return g_last_cuda_error; }

int pfb_pfaffian(int dtype, const void *A, int64_t batch, int n, int layout, void *out, void *stream)
{
    if (!valid_dtype(dtype) || !valid_layout(layout) || batch < 0 || n < 0) return PFB_ERR_INVALID;
    if (n > 32) return PFB_ERR_SIZE;
    if (batch == 0) return PFB_OK;
    if (!out || (!A && n > 0)) return PFB_ERR_INVALID;
    int rc = pfb::launch_small(dtype, false, A, batch, n, layout, out, nullptr, nullptr,
                               (cudaStream_t)stream);
    if (rc == PFB_ERR_CUDA) return cuda_failed();
    return rc;
}

size_t pfb_slog_workspace_bytes(int dtype, int64_t batch, int n, int mode)
{
    if (!valid_dtype(dtype) || batch < 0 || n < 0) return 0;
    if ((mode & 0xff) != PFB_MODE_FP64 && (mode & 0xff) != PFB_MODE_SPLIT) return 0;
    return pfb::large_workspace_bytes(dtype, batch, n, mode);
}

int pfb_slog_pfaffian(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                      double *log_out, void *sign_out, void *workspace, size_t workspace_bytes,
                      void *stream)
{
    return pfb_slog_pfaffian_timed(dtype, A, batch, n, layout, mode, log_out, sign_out, workspace,
                                   workspace_bytes, stream, nullptr);
}

int pfb_slog_max_concurrent(int dtype, int n)
{
    if (!valid_dtype(dtype) || n <= 32) return 0;
    return pfb::large_max_concurrent(dtype, n, PFB_PANEL_REGISTERS);
}

int pfb_slog_max_concurrent_form(int dtype, int n, int panel)
{
    if (!valid_dtype(dtype) || n <= 32 || (panel != PFB_PANEL_REGISTERS && panel != PFB_PANEL_HALF_SHARED)) return 0;
    pfb_slog_config over{panel, 0, 0, 0}, cf;
    if (!pfb::large_config(dtype, 1, n, PFB_MODE_FP64, &over, &cf)) return 0;
    return pfb::large_max_concurrent(dtype, n, panel);
}

int pfb_slog_config_for(int dtype, int64_t batch, int n, int mode, pfb_slog_config *out)
{
    if (!valid_dtype(dtype) || batch < 0 || n < 0 || !out) return PFB_ERR_INVALID;
    if (n <= 32 || (n & 1) || pfb::large_workspace_bytes(dtype, 1, n, mode) == 0) return PFB_ERR_SIZE;
    return pfb::large_config(dtype, batch, n, mode, nullptr, out) ? PFB_OK : PFB_ERR_INVALID;
}

int pfb_slog_stream_ranges(int dtype, int64_t batch, int n, int mode)
{
    pfb_slog_config cf;
    if (pfb_slog_config_for(dtype, batch, n, mode, &cf) != PFB_OK || batch <= 0) return 1;
    return pfb::large_second_range(dtype, batch, n, cf) > 0 ? 2 : 1;
}

int pfb_slog_panel_width(int dtype, int n)
{
    if (!valid_dtype(dtype) || n < 0) return 0;
    return pfb::large_panel_width(dtype, n);
}

int pfb_slog_pfaffian_timed(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                            double *log_out, void *sign_out, void *workspace, size_t workspace_bytes,
                            void *stream, const pfb_slog_timing *timing)
{
    return pfb_slog_pfaffian_ex(dtype, A, batch, n, layout, mode, log_out, sign_out, workspace, workspace_bytes,
                                stream, timing, nullptr);
}

int pfb_slog_pfaffian_ex(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                         double *log_out, void *sign_out, void *workspace, size_t workspace_bytes,
                         void *stream, const pfb_slog_timing *timing, const pfb_slog_config *config)
{
    if (!valid_dtype(dtype) || !valid_layout(layout) || batch < 0 || n < 0) return PFB_ERR_INVALID;
    if ((mode & 0xff) != PFB_MODE_FP64 && (mode & 0xff) != PFB_MODE_SPLIT) return PFB_ERR_INVALID;
    if ((mode & ~(0xfff | PFB_SPLIT_TEST_TIMEOUT)) != 0 || ((mode >> 8) & 0xf) > 7) return PFB_ERR_INVALID;
    if (batch == 0) return PFB_OK;
    if (!log_out || !sign_out || (!A && n > 0)) return PFB_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    if (n <= 32 || (n & 1)) {
        // odd orders give (-inf, 0) from the small kernel without reading A
        rc = pfb::launch_small(dtype, true, A, batch, (n & 1) ? 1 : n, layout, nullptr, log_out,
                               sign_out, s);
    } else {
        const size_t need = pfb::large_workspace_bytes(dtype, batch, n, mode);
        if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255u))
            return PFB_ERR_WORKSPACE;
        rc = pfb::launch_large(dtype, A, batch, n, layout, mode, log_out, sign_out, workspace,
                               workspace_bytes, s, timing, config);
    }
    if (rc == PFB_ERR_CUDA) return cuda_failed();
    return rc;
}

int pfb_slog_pfaffian_ptrs(int dtype, const void *const *A_ptrs, int64_t batch, int n, int layout, int mode,
                           double *log_out, void *sign_out, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!valid_dtype(dtype) || !valid_layout(layout) || batch < 0 || n < 0) return PFB_ERR_INVALID;
    if ((mode & 0xff) != PFB_MODE_FP64 && (mode & 0xff) != PFB_MODE_SPLIT) return PFB_ERR_INVALID;
    if ((mode & ~0xfff) != 0 || ((mode >> 8) & 0xf) > 7) return PFB_ERR_INVALID;
    if (n <= 32 || (n & 1)) return PFB_ERR_SIZE;
    if (batch == 0) return PFB_OK;
    if (!A_ptrs || !log_out || !sign_out) return PFB_ERR_INVALID;
    const size_t need = pfb::large_workspace_bytes(dtype, batch, n, mode);
    if (need == 0) return PFB_ERR_SIZE;
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255u)) return PFB_ERR_WORKSPACE;
    const int rc = pfb::launch_large(dtype, nullptr, batch, n, layout, mode, log_out, sign_out, workspace,
                                     workspace_bytes, (cudaStream_t)stream, nullptr, nullptr, A_ptrs);
    if (rc == PFB_ERR_CUDA) return cuda_failed();
    return rc;
}

size_t pfb_slog_grad_workspace_bytes(int dtype, int64_t batch, int n, int mode)
{
    if (!valid_dtype(dtype) || batch < 0 || n < 2 || (n & 1)) return 0;
    return pfb::grad_workspace_bytes(dtype, batch, n, mode);
}

int pfb_slog_pfaffian_grad(int dtype, const void *A, int64_t batch, int n, int layout, int mode,
                           const double *ct_log, void *G_out, double *log_out, void *sign_out,
                           void *workspace, size_t workspace_bytes, void *stream)
{
    if (!valid_dtype(dtype) || !valid_layout(layout) || batch < 0 || n < 0) return PFB_ERR_INVALID;
    if ((mode & 0xff) != PFB_MODE_FP64 && (mode & 0xff) != PFB_MODE_SPLIT) return PFB_ERR_INVALID;
    if ((mode & ~(0xfff | PFB_SPLIT_TEST_TIMEOUT)) != 0 || ((mode >> 8) & 0xf) > 7) return PFB_ERR_INVALID;
    if (n < 2 || (n & 1)) return PFB_ERR_SIZE;
    if (batch == 0) return PFB_OK;
    if (!A || !G_out || !log_out || !sign_out) return PFB_ERR_INVALID;
    const size_t need1 = pfb::grad_workspace_bytes(dtype, 1, n, mode);   // one matrix at a time
    if (need1 == 0) return PFB_ERR_SIZE;
    if (!workspace || workspace_bytes < need1 || ((uintptr_t)workspace & 255u)) return PFB_ERR_WORKSPACE;
    const int rc = pfb::launch_grad(dtype, A, batch, n, layout, mode, ct_log, G_out, log_out, sign_out,
                                    workspace, workspace_bytes, (cudaStream_t)stream);
    if (rc == PFB_ERR_CUDA) return cuda_failed();
    return rc;
}

size_t pfb_slog_ragged_workspace_bytes(int64_t count, int max_n)
{
    return pfb::ragged_workspace_bytes(count, max_n);
}

int pfb_slog_pfaffian_ragged(const void *const *A, const int32_t *n, const int32_t *dtype, int64_t count,
                             int max_n, int layout, double *log_out, double *sign_out, void *workspace,
                             size_t workspace_bytes, void *stream)
{
    if (count < 0 || max_n < 0 || !valid_layout(layout)) return PFB_ERR_INVALID;
    if (max_n > PFB_RAGGED_MAX_N) return PFB_ERR_SIZE;
    if (count == 0) return PFB_OK;
    if (!A || !n || !dtype || !log_out || !sign_out) return PFB_ERR_INVALID;
    const size_t need = pfb::ragged_workspace_bytes(count, max_n);
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255u)) return PFB_ERR_WORKSPACE;
    const int rc = pfb::launch_ragged(A, n, dtype, count, max_n, layout, log_out, sign_out, workspace,
                                      (cudaStream_t)stream);
    if (rc == PFB_ERR_CUDA) return cuda_failed();
    return rc;
}

size_t pfb_upload_upper_bytes(int dtype, int64_t batch, int n)
{
    if (!valid_dtype(dtype) || batch < 0 || n < 0) return 0;
    const size_t es = dtype_bytes(dtype);
    if (n <= 32) return (size_t)batch * (size_t)n * (size_t)n * es;
    size_t per = 0;
    for (int r0 = 0; r0 < n; r0 += kUploadRows) {
        const int rows = n - r0 < kUploadRows ? n - r0 : kUploadRows;
        per += (size_t)rows * (size_t)(n - r0) * es;
    }
    return per * (size_t)batch;
}

int pfb_upload_upper(int dtype, const void *A_host, void *A_dev, int64_t batch, int n, void *stream)
{
    if (!valid_dtype(dtype) || batch < 0 || n < 0) return PFB_ERR_INVALID;
    if (batch == 0 || n == 0) return PFB_OK;
    if (!A_host || !A_dev) return PFB_ERR_INVALID;
    const cudaStream_t s = (cudaStream_t)stream;
    const size_t es = dtype_bytes(dtype);
    const size_t pitch = (size_t)n * es, mat = (size_t)n * pitch;
    if (n <= 32)
        return cuda_status(cudaMemcpyAsync(A_dev, A_host, (size_t)batch * mat, cudaMemcpyHostToDevice, s));
    const char *src = static_cast<const char *>(A_host);
    char *dst = static_cast<char *>(A_dev);
    for (int64_t b = 0; b < batch; b++)
        for (int r0 = 0; r0 < n; r0 += kUploadRows) {
            const int rows = n - r0 < kUploadRows ? n - r0 : kUploadRows;
            const size_t off = (size_t)b * mat + (size_t)r0 * pitch + (size_t)r0 * es;
            const cudaError_t e = cudaMemcpy2DAsync(dst + off, pitch, src + off, pitch, (size_t)(n - r0) * es,
                                                    (size_t)rows, cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return cuda_status(e);
        }
    return PFB_OK;
}

int pfb_slog_pivots(int64_t batch, int n, const void *workspace, size_t workspace_bytes,
                    int32_t *piv_out, void *stream)
{
    if (batch < 0 || n < 0 || !piv_out || !workspace) return PFB_ERR_INVALID;
    return pfb::large_copy_pivots(batch, n, workspace, workspace_bytes, piv_out, (cudaStream_t)stream);
}

}  // extern "C"
