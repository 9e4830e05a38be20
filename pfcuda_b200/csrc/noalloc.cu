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
// address, so its device address is looked up once per device (with that
// device current) by cudaGetSymbolAddress on the first call made on the device,
// and that address is what the kernels are given.
//
// All calls share the array, and it keeps the last call's contents.  Nothing of
// it has to start at zero: the factorisation's first kernel overwrites the
// working matrix and the per-matrix state it later reads, and every pivot is
// written before it is read.  Calls whose work overlaps on the GPU (two streams,
// or two host threads) race on the array and must be serialised by the caller.
#include <mutex>

#include "common.cuh"
#include "small.cuh"
#include "large.cuh"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[PFB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices];

// Device address of g_noalloc_scratch on the current device (looked up once).
int scratch_address(void **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PFB_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return PFB_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PFB_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
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
