// noalloc.cu -- pfb_slog_pfaffian_noalloc: the large-matrix (log|Pf|, sign) path
// with its scratch memory inside the library instead of a caller workspace.
//
// Some callers cannot allocate device memory: a plugin that is handed raw
// device pointers by a host framework that owns every allocation (and gives the
// plugin no allocator), a binding from a host language with no CUDA allocator
// wired in, or a latency-critical path where a cudaMalloc -- which may
// synchronise the whole device -- is not acceptable.  For them the workspace of
// pfb_slog_pfaffian lives in one file-scope device array, g_noalloc_scratch,
// of PFB_NOALLOC_SCRATCH_BYTES.  Every GPU that loads this library holds that
// array until the process exits.
//
// In host code the array's name is only a host-side stand-in, never a device
// address, so every call looks up its device address on the current device
// with cudaGetSymbolAddress (a cheap query once the module is loaded) and
// hands that address to the kernels.  Nothing is cached, so a device reset or
// a new context between calls cannot leave a stale address behind.  The first
// call on a device loads the library's module there, so make that first call
// before any stream capture.
//
// All calls share the array, and it keeps the last call's contents.  Nothing of
// it has to start at zero: the factorisation's first kernel overwrites the
// working matrix and the per-matrix state it later reads, and every pivot is
// written before it is read.  Calls whose work overlaps on the GPU (two streams,
// or two host threads) race on the array and must be serialised by the caller.
#include "common.cuh"
#include "small.cuh"
#include "large.cuh"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[PFB_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device.
int scratch_address(void **out)
{
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PFB_ERR_CUDA;
    *out = p;
    return PFB_OK;
}

}  // namespace

extern "C" int pfb_slog_pfaffian_noalloc(int dtype, const void *A, int64_t batch, int n, int layout,
                                         int mode, double *log_out, void *sign_out, void *stream)
{
    if (dtype < PFB_F32 || dtype > PFB_C128 || (layout != PFB_ROW_MAJOR && layout != PFB_COL_MAJOR) ||
        batch < 0 || n < 0)
        return PFB_ERR_INVALID;
    if ((mode & 0xff) != PFB_MODE_FP64 && (mode & 0xff) != PFB_MODE_SPLIT) return PFB_ERR_INVALID;
    if (batch == 0) return PFB_OK;
    if (!log_out || !sign_out || (!A && n > 0)) return PFB_ERR_INVALID;
    if (n <= 32 || (n & 1)) {
        // the small kernel needs no scratch at all
        return pfb_slog_pfaffian(dtype, A, batch, n, layout, mode, log_out, sign_out, nullptr, 0, stream);
    }
    const size_t need = pfb_slog_workspace_bytes(dtype, batch, n, mode);
    if (need == 0 || need > (size_t)PFB_NOALLOC_SCRATCH_BYTES) return PFB_ERR_SIZE;
    void *scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc != PFB_OK) return rc;
    return pfb_slog_pfaffian(dtype, A, batch, n, layout, mode, log_out, sign_out, scratch,
                             (size_t)PFB_NOALLOC_SCRATCH_BYTES, stream);
}
