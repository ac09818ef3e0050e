// dual.cuh — forward-mode dual numbers for the adjoint of the step.
//
// D2 carries a value and its derivatives along two input directions.  The
// value is computed with exactly the float operation the plain code performs
// (same rounding), so running the templated physics (physics.cuh) on D2
// reproduces the float results bit for bit while the tangents give the
// local Jacobian.
//
// Only the value needs the plain code's rounding: the tangents use the fast
// reciprocal-based division (__fdividef, within 2 ulp), which is far cheaper
// than an IEEE division and accurate well beyond what a derivative needs.
//
// Derivatives at kinks (the subgradient chosen):
//   xmax(x, c)        derivative of x when x > c, else 0
//   xclamp(x, lo, hi) derivative of x when lo < x < hi, else 0
//   xabs(x)           sign(x) * derivative (0 at x == 0)
//   sqrt, cbrt, pow   0 where the input tangent is 0 (no 0 * inf at x == 0)
// and branch tests (regime, reflection, ratio < 0.5) read the value only.
#pragma once

#include <cuda_runtime.h>

namespace fpg {

struct D2 {
    float v, a, b;
    __device__ __forceinline__ D2() : v(0.0f), a(0.0f), b(0.0f) {}
    __device__ __forceinline__ D2(float x) : v(x), a(0.0f), b(0.0f) {}
    __device__ __forceinline__ D2(float x, float da, float db) : v(x), a(da), b(db) {}
};

__device__ __forceinline__ float val(const D2& x) { return x.v; }

__device__ __forceinline__ D2 operator-(const D2& x) { return D2(-x.v, -x.a, -x.b); }
__device__ __forceinline__ D2 operator+(const D2& x, const D2& y) { return D2(x.v + y.v, x.a + y.a, x.b + y.b); }
__device__ __forceinline__ D2 operator+(const D2& x, float c) { return D2(x.v + c, x.a, x.b); }
__device__ __forceinline__ D2 operator+(float c, const D2& x) { return D2(c + x.v, x.a, x.b); }
__device__ __forceinline__ D2 operator-(const D2& x, const D2& y) { return D2(x.v - y.v, x.a - y.a, x.b - y.b); }
__device__ __forceinline__ D2 operator-(const D2& x, float c) { return D2(x.v - c, x.a, x.b); }
__device__ __forceinline__ D2 operator-(float c, const D2& x) { return D2(c - x.v, -x.a, -x.b); }
__device__ __forceinline__ D2 operator*(const D2& x, const D2& y) {
    return D2(x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b);
}
__device__ __forceinline__ D2 operator*(const D2& x, float c) { return D2(x.v * c, x.a * c, x.b * c); }
__device__ __forceinline__ D2 operator*(float c, const D2& x) { return D2(c * x.v, c * x.a, c * x.b); }
// The value is the step's division (sdiv), as in the float code.
__device__ __forceinline__ D2 operator/(const D2& x, const D2& y) {
    const float q = sdiv(x.v, y.v);
    const float r = __fdividef(1.0f, y.v);
    return D2(q, (x.a - q * y.a) * r, (x.b - q * y.b) * r);
}
__device__ __forceinline__ D2 operator/(const D2& x, float c) {
    const float r = __fdividef(1.0f, c);
    return D2(sdiv(x.v, c), x.a * r, x.b * r);
}
__device__ __forceinline__ D2 operator/(float c, const D2& y) {
    const float q = sdiv(c, y.v);
    const float r = -q * __fdividef(1.0f, y.v);
    return D2(q, r * y.a, r * y.b);
}

__device__ __forceinline__ D2 xdiv(const D2& x, const D2& y) { return x / y; }
__device__ __forceinline__ D2 xdiv(const D2& x, float c) { return x / c; }
__device__ __forceinline__ D2 xdiv(float c, const D2& y) { return c / y; }

__device__ __forceinline__ D2 xexp(const D2& x) {
    const float e = xexp(x.v);
    return D2(e, e * x.a, e * x.b);
}
__device__ __forceinline__ D2 xsqrt(const D2& x) {
    const float s = sqrtf(x.v);
    const float k = __fdividef(0.5f, s);
    return D2(s, x.a == 0.0f ? 0.0f : x.a * k, x.b == 0.0f ? 0.0f : x.b * k);
}
__device__ __forceinline__ D2 xcbrt(const D2& x) {
    const float c = cbrtf(x.v);
    const float k = __fdividef(1.0f, 3.0f * c * c);
    return D2(c, x.a == 0.0f ? 0.0f : x.a * k, x.b == 0.0f ? 0.0f : x.b * k);
}
__device__ __forceinline__ D2 xpow(const D2& x, float e) {
    const float p = pow_pos(x.v, e);
    const float k = __fdividef(e * p, x.v);
    return D2(p, x.a == 0.0f ? 0.0f : x.a * k, x.b == 0.0f ? 0.0f : x.b * k);
}
__device__ __forceinline__ D2 xmax(const D2& x, float c) {
    return x.v > c ? x : D2(fmaxf(x.v, c));
}
__device__ __forceinline__ D2 xclamp(const D2& x, float lo, float hi) {
    const float v = fminf(fmaxf(x.v, lo), hi);
    return (x.v > lo && x.v < hi) ? D2(v, x.a, x.b) : D2(v);
}
__device__ __forceinline__ D2 xabs(const D2& x) {
    return x.v > 0.0f ? x : x.v < 0.0f ? -x : D2(fabsf(x.v));
}

}  // namespace fpg
