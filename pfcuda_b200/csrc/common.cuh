// common.cuh -- scalar types, complex arithmetic and warp helpers shared by the
// engine's kernels.
//
// The reference's type layer (include/pfaffian_utils.cuh:10-72) maps each dtype
// to a cuComplex-based scalar with a real "projection" type and a magnitude.
// The same roles here: Scalar<T> (storage type -> compute ops), RealOf<T>, and
// mag() (the modulus used for pivot selection, hypot for complex as
// numpy.abs does).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <type_traits>

#include "../../include/pfb200.h"

#define PFB_HD __host__ __device__ __forceinline__
#define PFB_D __device__ __forceinline__

namespace pfb {

template <typename R>
struct __align__(2 * sizeof(R)) cplx {
    R re, im;
};

using c64 = cplx<float>;
using c128 = cplx<double>;

template <typename T> struct RealOf { using type = T; };
template <typename R> struct RealOf<cplx<R>> { using type = R; };

template <typename T> struct IsComplex { static constexpr bool value = false; };
template <typename R> struct IsComplex<cplx<R>> { static constexpr bool value = true; };

// ---------------------------------------------------------------- arithmetic

template <typename R> PFB_HD cplx<R> mk(R re, R im) { cplx<R> z; z.re = re; z.im = im; return z; }

template <typename R> PFB_HD cplx<R> operator+(cplx<R> a, cplx<R> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename R> PFB_HD cplx<R> operator-(cplx<R> a, cplx<R> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename R> PFB_HD cplx<R> operator-(cplx<R> a) { return mk(-a.re, -a.im); }
template <typename R> PFB_HD cplx<R> operator*(cplx<R> a, cplx<R> b)
{
    return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename R> PFB_HD bool operator==(cplx<R> a, cplx<R> b) { return a.re == b.re && a.im == b.im; }

template <typename T> PFB_HD T zero() { return T(0); }
template <> PFB_HD c64 zero<c64>() { return mk(0.f, 0.f); }
template <> PFB_HD c128 zero<c128>() { return mk(0.0, 0.0); }
template <typename T> PFB_HD T one() { return T(1); }
template <> PFB_HD c64 one<c64>() { return mk(1.f, 0.f); }
template <> PFB_HD c128 one<c128>() { return mk(1.0, 0.0); }

PFB_HD bool is_zero(float x) { return x == 0.f; }
PFB_HD bool is_zero(double x) { return x == 0.0; }
template <typename R> PFB_HD bool is_zero(cplx<R> x) { return x.re == R(0) && x.im == R(0); }

// acc + a*b and acc - a*b with fused multiply-adds
PFB_HD float fma_(float a, float b, float c) { return fmaf(a, b, c); }
PFB_HD double fma_(double a, double b, double c) { return fma(a, b, c); }
template <typename R> PFB_HD cplx<R> fma_(cplx<R> a, cplx<R> b, cplx<R> c)
{
    return mk(fma_(-a.im, b.im, fma_(a.re, b.re, c.re)), fma_(a.im, b.re, fma_(a.re, b.im, c.im)));
}
// c - a*b
PFB_HD float fms_(float a, float b, float c) { return fmaf(-a, b, c); }
PFB_HD double fms_(double a, double b, double c) { return fma(-a, b, c); }
template <typename R> PFB_HD cplx<R> fms_(cplx<R> a, cplx<R> b, cplx<R> c)
{
    return mk(fma_(a.im, b.im, fma_(-a.re, b.re, c.re)), fma_(-a.im, b.re, fma_(-a.re, b.im, c.im)));
}

// 1/a
PFB_HD float recip(float a) { return 1.f / a; }
PFB_HD double recip(double a) { return 1.0 / a; }
template <typename R> PFB_HD cplx<R> recip(cplx<R> a)
{
    // Smith-style scaling keeps |a|^2 from overflowing or underflowing.
    R s = fabs(a.re) >= fabs(a.im) ? a.re : a.im;
    if (s == R(0)) return mk(R(1) / s, R(0));
    R ar = a.re / s, ai = a.im / s;
    R d = (ar * a.re + ai * a.im);
    return mk(ar / d, -ai / d);
}

// modulus used for pivoting (numpy.abs semantics: hypot for complex)
PFB_HD float mag(float x) { return fabsf(x); }
PFB_HD double mag(double x) { return fabs(x); }
PFB_HD float mag(c64 x) { return hypotf(x.re, x.im); }
PFB_HD double mag(c128 x) { return hypot(x.re, x.im); }

// scale by a real
PFB_HD float scal(float a, float s) { return a * s; }
PFB_HD double scal(double a, double s) { return a * s; }
template <typename R> PFB_HD cplx<R> scal(cplx<R> a, R s) { return mk(a.re * s, a.im * s); }

// conversions between storage and compute types
template <typename To, typename From> struct Conv;
template <typename T> struct Conv<T, T> { static PFB_HD T f(T x) { return x; } };
template <> struct Conv<double, float> { static PFB_HD double f(float x) { return (double)x; } };
template <> struct Conv<float, double> { static PFB_HD float f(double x) { return (float)x; } };
template <> struct Conv<c128, c64> { static PFB_HD c128 f(c64 x) { return mk((double)x.re, (double)x.im); } };
template <> struct Conv<c64, c128> { static PFB_HD c64 f(c128 x) { return mk((float)x.re, (float)x.im); } };
template <typename To, typename From> PFB_HD To conv(From x) { return Conv<To, From>::f(x); }

// ---------------------------------------------------------------- shuffles

PFB_D float shfl(float v, int src, int width = 32) { return __shfl_sync(0xffffffffu, v, src, width); }
PFB_D double shfl(double v, int src, int width = 32) { return __shfl_sync(0xffffffffu, v, src, width); }
PFB_D int shfl(int v, int src, int width = 32) { return __shfl_sync(0xffffffffu, v, src, width); }
template <typename R> PFB_D cplx<R> shfl(cplx<R> v, int src, int width = 32)
{
    return mk(shfl(v.re, src, width), shfl(v.im, src, width));
}
PFB_D float shfl_xor(float v, int m, int width = 32) { return __shfl_xor_sync(0xffffffffu, v, m, width); }
PFB_D double shfl_xor(double v, int m, int width = 32) { return __shfl_xor_sync(0xffffffffu, v, m, width); }
PFB_D int shfl_xor(int v, int m, int width = 32) { return __shfl_xor_sync(0xffffffffu, v, m, width); }

// Compile-time loop: f(std::integral_constant<int, i>) for i = I, I+S, ... < E.
// Register arrays indexed by i stay in registers, whatever the unroller decides.
template <int I, int E, int S, typename F>
PFB_D void static_for(F &&f)
{
    if constexpr (I < E) {
        f(std::integral_constant<int, I>{});
        static_for<I + S, E, S>(f);
    }
}

// read-only global loads
PFB_D float ldg(const float *p) { return __ldg(p); }
PFB_D double ldg(const double *p) { return __ldg(p); }
PFB_D c64 ldg(const c64 *p)
{
    float2 v = __ldg(reinterpret_cast<const float2 *>(p));
    return mk(v.x, v.y);
}
PFB_D c128 ldg(const c128 *p)
{
    double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return mk(v.x, v.y);
}

// The CUDA error of the calling host thread's most recent failing call (what
// pfb_last_cuda_error returns); defined in capi.cu.
int &last_cuda_error();

// PFB_OK, or PFB_ERR_CUDA with the error recorded, for a runtime call's result.
inline int cuda_check(cudaError_t e)
{
    if (e == cudaSuccess) return PFB_OK;
    last_cuda_error() = (int)e;
    return PFB_ERR_CUDA;
}
// The same for the launches just made (cudaGetLastError clears a launch error,
// so it is recorded here, where it is read).
inline int launch_status() { return cuda_check(cudaGetLastError()); }

// dtype enum -> storage type
template <int D> struct DT;
template <> struct DT<PFB_F32> { using type = float; };
template <> struct DT<PFB_F64> { using type = double; };
template <> struct DT<PFB_C64> { using type = c64; };
template <> struct DT<PFB_C128> { using type = c128; };

inline size_t dtype_size(int dt)
{
    switch (dt) {
    case PFB_F32: return 4;
    case PFB_F64: return 8;
    case PFB_C64: return 8;
    case PFB_C128: return 16;
    default: return 0;
    }
}

}  // namespace pfb
