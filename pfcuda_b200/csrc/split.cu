// split.cu -- split-precision trailing update (int8 slices, tcgen05).
#include "split.cuh"
#include "large.cuh"

namespace pfb {

bool split_available() { return false; }

size_t split_workspace_bytes(bool cplx, int64_t batch, int n, int nb)
{
    const int kk = cplx ? 2 * nb : nb;
    const int slices = 7;
    return (size_t)batch * ((size_t)2 * slices * n * kk + (size_t)n * 4) + 1024;
}

SplitArgs split_args(bool use, unsigned char *ws, bool cplx, int64_t batch, int n, int nb, int k0)
{
    SplitArgs a{};
    a.enabled = use ? 1 : 0;
    a.n = n;
    a.k0 = k0;
    a.nb = nb;
    a.kk = cplx ? 2 * nb : nb;
    a.slices = 7;
    a.mstride = (int64_t)a.slices * n * a.kk;
    a.xs = reinterpret_cast<int8_t *>(ws);
    a.ys = a.xs + batch * a.mstride;
    a.ex = reinterpret_cast<int32_t *>(a.ys + batch * a.mstride);
    return a;
}

int launch_split_update(bool, void *, int, int, int, int64_t, const MatState *, const SplitArgs &,
                        cudaStream_t)
{
    return PFB_ERR_UNSUPPORTED;
}

}  // namespace pfb
