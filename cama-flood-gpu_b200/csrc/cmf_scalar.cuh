// Scalar layer of the routing physics.
//
// The per-element physics (cmf_physics.cuh) is written once, as templates on
// its scalar types, and instantiated three ways:
//
//   float / double   the forward kernels (cmf_device.cuh): plain IEEE
//                    arithmetic, CUDA's fmax/fmin/sqrt/cbrt/exp/log;
//   double, Dual     the adjoint (cmf_adjoint.cu): its primal on double and
//                    its Jacobian columns on Dual, a forward-mode dual number
//                    (value and one directional derivative), or on DualN<K>
//                    (value and K directional derivatives in one pass).
//
// Conventions of the Dual operations (those of the PyTorch transcription the
// adjoint is checked against, for the branches evaluated this way): smax and
// smin pass the derivative of the first operand on a tie; ssqrt and scbrt
// have derivative 0 at 0; sabs has derivative 0 at 0.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace cmf {

struct Dual {
    double v, d;
    Dual() = default;
    __host__ __device__ constexpr Dual(double value) : v(value), d(0.0) {}
    __host__ __device__ constexpr Dual(double value, double deriv) : v(value), d(deriv) {}
};

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b)
{
    const double q = a / b.v;
    return {q, -q * b.d / b.v};
}

// value of a scalar (the primal value of a Dual); used for every comparison,
// so branch decisions never depend on a derivative
__device__ __forceinline__ float val(float x) { return x; }
__device__ __forceinline__ double val(double x) { return x; }
__device__ __forceinline__ double val(const Dual& x) { return x.v; }

__device__ __forceinline__ float smax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double smax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ Dual smax(Dual a, Dual b) { return a.v >= b.v ? a : b; }
__device__ __forceinline__ float smin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double smin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ Dual smin(Dual a, Dual b) { return a.v <= b.v ? a : b; }

__device__ __forceinline__ float ssqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double ssqrt(double a) { return sqrt(a); }
__device__ __forceinline__ Dual ssqrt(Dual a)
{
    const double s = sqrt(a.v);
    return {s, a.v > 0.0 ? a.d / (2.0 * s) : 0.0};
}
__device__ __forceinline__ float scbrt(float a) { return cbrtf(a); }
__device__ __forceinline__ double scbrt(double a) { return cbrt(a); }
__device__ __forceinline__ Dual scbrt(Dual a)
{
    const double c = cbrt(a.v);
    return {c, a.v != 0.0 ? a.d / (3.0 * c * c) : 0.0};
}
__device__ __forceinline__ float sexp(float a) { return expf(a); }
__device__ __forceinline__ double sexp(double a) { return exp(a); }
__device__ __forceinline__ Dual sexp(Dual a)
{
    const double e = exp(a.v);
    return {e, e * a.d};
}
__device__ __forceinline__ float slog(float a) { return logf(a); }
__device__ __forceinline__ double slog(double a) { return log(a); }
__device__ __forceinline__ Dual slog(Dual a) { return {log(a.v), a.d / a.v}; }
__device__ __forceinline__ float sabs(float a) { return fabsf(a); }
__device__ __forceinline__ double sabs(double a) { return fabs(a); }
__device__ __forceinline__ Dual sabs(Dual a)
{
    return {fabs(a.v), (double)((a.v > 0.0) - (a.v < 0.0)) * a.d};
}

// Rounded operations with the contraction fixed: fused multiply-add where
// the expression has one, separately rounded products and sums elsewhere.
// Code written with them rounds the same however the compiler arranges the
// surrounding control flow (branches, sunk or hoisted values); on Dual they
// are the plain operations.
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ Dual xfma(Dual a, Dual b, Dual c) { return a * b + c; }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ Dual xmul(Dual a, Dual b) { return a * b; }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ Dual xadd(Dual a, Dual b) { return a + b; }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ Dual xsub(Dual a, Dual b) { return a - b; }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ Dual xdiv(Dual a, Dual b) { return a / b; }

// ---------------------------------------------------------------------------
// DualN<K>: a value and K directional derivatives, carried through one
// evaluation.  A Jacobian-vector product over K input directions then costs
// one pass whose primal part (the divisions, roots and branches) runs once
// instead of K times.  Same conventions as Dual; quotients scale the
// derivatives by one reciprocal of the divisor.
// ---------------------------------------------------------------------------
template <int K>
struct DualN {
    double v;
    double d[K];
    DualN() = default;
    __host__ __device__ constexpr DualN(double value) : v(value), d{} {}
};

template <int K>
__device__ __forceinline__ DualN<K> scaled(const DualN<K>& a, double value, double f)
{
    DualN<K> r;
    r.v = value;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * f;
    return r;
}

template <int K>
__device__ __forceinline__ DualN<K> operator+(const DualN<K>& a, const DualN<K>& b)
{
    DualN<K> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ DualN<K> operator-(const DualN<K>& a, const DualN<K>& b)
{
    DualN<K> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ DualN<K> operator-(const DualN<K>& a) { return scaled(a, -a.v, -1.0); }
template <int K>
__device__ __forceinline__ DualN<K> operator*(const DualN<K>& a, const DualN<K>& b)
{
    DualN<K> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ DualN<K> operator/(const DualN<K>& a, const DualN<K>& b)
{
    DualN<K> r;
    r.v = a.v / b.v;
    const double inv = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
template <int K>
__device__ __forceinline__ DualN<K> operator+(const DualN<K>& a, double b)
{
    DualN<K> r = a;
    r.v = a.v + b;
    return r;
}
template <int K>
__device__ __forceinline__ DualN<K> operator+(double a, const DualN<K>& b) { return b + a; }
template <int K>
__device__ __forceinline__ DualN<K> operator-(const DualN<K>& a, double b)
{
    DualN<K> r = a;
    r.v = a.v - b;
    return r;
}
template <int K>
__device__ __forceinline__ DualN<K> operator-(double a, const DualN<K>& b) { return scaled(b, a - b.v, -1.0); }
template <int K>
__device__ __forceinline__ DualN<K> operator*(const DualN<K>& a, double b) { return scaled(a, a.v * b, b); }
template <int K>
__device__ __forceinline__ DualN<K> operator*(double a, const DualN<K>& b) { return scaled(b, a * b.v, a); }
template <int K>
__device__ __forceinline__ DualN<K> operator/(const DualN<K>& a, double b) { return scaled(a, a.v / b, 1.0 / b); }
template <int K>
__device__ __forceinline__ DualN<K> operator/(double a, const DualN<K>& b)
{
    const double q = a / b.v;
    return scaled(b, q, -q / b.v);
}

template <int K>
__device__ __forceinline__ double val(const DualN<K>& x) { return x.v; }
template <int K>
__device__ __forceinline__ DualN<K> smax(const DualN<K>& a, const DualN<K>& b) { return a.v >= b.v ? a : b; }
template <int K>
__device__ __forceinline__ DualN<K> smin(const DualN<K>& a, const DualN<K>& b) { return a.v <= b.v ? a : b; }
template <int K>
__device__ __forceinline__ DualN<K> ssqrt(const DualN<K>& a)
{
    const double s = sqrt(a.v);
    return scaled(a, s, a.v > 0.0 ? 0.5 / s : 0.0);
}
template <int K>
__device__ __forceinline__ DualN<K> scbrt(const DualN<K>& a)
{
    const double c = cbrt(a.v);
    return scaled(a, c, a.v != 0.0 ? 1.0 / (3.0 * c * c) : 0.0);
}
template <int K>
__device__ __forceinline__ DualN<K> sexp(const DualN<K>& a)
{
    const double e = exp(a.v);
    return scaled(a, e, e);
}
template <int K>
__device__ __forceinline__ DualN<K> slog(const DualN<K>& a) { return scaled(a, log(a.v), 1.0 / a.v); }
template <int K>
__device__ __forceinline__ DualN<K> sabs(const DualN<K>& a)
{
    return scaled(a, fabs(a.v), (double)((a.v > 0.0) - (a.v < 0.0)));
}
template <int K>
__device__ __forceinline__ DualN<K> xfma(const DualN<K>& a, const DualN<K>& b, const DualN<K>& c) { return a * b + c; }
template <int K>
__device__ __forceinline__ DualN<K> xmul(const DualN<K>& a, const DualN<K>& b) { return a * b; }
template <int K>
__device__ __forceinline__ DualN<K> xadd(const DualN<K>& a, const DualN<K>& b) { return a + b; }
template <int K>
__device__ __forceinline__ DualN<K> xsub(const DualN<K>& a, const DualN<K>& b) { return a - b; }
template <int K>
__device__ __forceinline__ DualN<K> xdiv(const DualN<K>& a, const DualN<K>& b) { return a / b; }

// positive part, written as the comparison the storage clips use (a NaN or a
// negative zero becomes +0)
template <typename T>
__device__ __forceinline__ T pos_part(T x) { return val(x) > 0 ? x : T(0); }

// a storage-typed value narrowed to the flux type (a no-op for Dual)
template <typename To, typename From>
__device__ __forceinline__ To narrow(From x) { return static_cast<To>(x); }

}  // namespace cmf
