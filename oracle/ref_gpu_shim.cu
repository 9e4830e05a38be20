// ref_gpu_shim.cu -- C entry points over the reference's own CUDA launchers.
//
// TEST INFRASTRUCTURE ONLY.  Compiled with the UNMODIFIED reference sources
// src/pfaffian.cu, src/pfaffian_sm.cu, src/slog_pfaffian.cu and
// src/slog_pfaffian_lg.cu (read where they lie) into oracle/_ref/libref_gpu.so,
// so that the reference GPU kernels can be run on the same inputs as this engine
// without JAX.  It replays what the reference's XLA handlers do
// (bindings/jax_bindings.cu:19-112): one launcher call per matrix on one
// stream, and for slog a device copy of each matrix first because the
// reference algorithm overwrites it (jax_bindings.cu:52-72).
//
// Each matrix is passed the way XLA hands it to the reference, column-major
// (pfcuda/cuda_api.py:50 input_layouts=[(1, 0)]); the kernels index it with
// CM(A, n, r, c) = A[r + c*n] (include/pfaffian_utils.cuh:10).
#include <cstdint>
#include <stdexcept>
#include "pfaffian.cuh"
#include "slog_pfaffian_lg.cuh"

template <typename T>
static int run_pf(const void* dA, int64_t B, int n, void* dOut, cudaStream_t s)
{
    try {
        const T* A = static_cast<const T*>(dA);
        T* out = static_cast<T*>(dOut);
        for (int64_t b = 0; b < B; b++)
            pfaffian<T>(A + (size_t)b * n * n, (unsigned)n, out + b, s);
    } catch (const std::exception&) {
        return 1;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

template <typename T>
static int run_slog(const void* dA, int64_t B, int n, void* dLog, void* dPhase,
                    void* dTmp, cudaStream_t s)
{
    using R = typename ProjectionType<T>::type;
    const T* A = static_cast<const T*>(dA);
    T* tmp = static_cast<T*>(dTmp);
    for (int64_t b = 0; b < B; b++) {
        if (cudaMemcpyAsync(tmp, A + (size_t)b * n * n, sizeof(T) * (size_t)n * n,
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return 2;
        slog_pfaffian_lg<T>(tmp, (unsigned)n, static_cast<R*>(dLog) + b,
                            static_cast<T*>(dPhase) + b, s);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" {
int refgpu_pfaffian_f32(const void* A, int64_t B, int n, void* o, cudaStream_t s) { return run_pf<float>(A, B, n, o, s); }
int refgpu_pfaffian_f64(const void* A, int64_t B, int n, void* o, cudaStream_t s) { return run_pf<double>(A, B, n, o, s); }
int refgpu_pfaffian_c64(const void* A, int64_t B, int n, void* o, cudaStream_t s) { return run_pf<cuFloatComplex>(A, B, n, o, s); }
int refgpu_pfaffian_c128(const void* A, int64_t B, int n, void* o, cudaStream_t s) { return run_pf<cuDoubleComplex>(A, B, n, o, s); }
// log is float for f32/c64 and double for f64/c128 (ProjectionType, pfaffian_utils.cuh:13-15)
int refgpu_slog_f32(const void* A, int64_t B, int n, void* l, void* p, void* t, cudaStream_t s) { return run_slog<float>(A, B, n, l, p, t, s); }
int refgpu_slog_f64(const void* A, int64_t B, int n, void* l, void* p, void* t, cudaStream_t s) { return run_slog<double>(A, B, n, l, p, t, s); }
int refgpu_slog_c64(const void* A, int64_t B, int n, void* l, void* p, void* t, cudaStream_t s) { return run_slog<cuFloatComplex>(A, B, n, l, p, t, s); }
int refgpu_slog_c128(const void* A, int64_t B, int n, void* l, void* p, void* t, cudaStream_t s) { return run_slog<cuDoubleComplex>(A, B, n, l, p, t, s); }
}
