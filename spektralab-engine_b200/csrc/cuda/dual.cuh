// Forward-mode dual numbers for the render's adjoint (vjp.cu): a binary32 value and N tangents.
//
// The per-pixel stages of the render (expose, develop with the grain held fixed, print) map a few inputs
// to a few outputs. Evaluated on Dual<N> with one tangent per input (and per scalar parameter), a stage
// yields its Jacobian at the pixel, and the vector-Jacobian product is the upstream gradient times it.
// Non-smooth operations take the derivative of the branch the value takes: max/min/clamp pass the
// selected argument's tangent, floor and comparisons carry none, a lookup carries the slope of the
// interval the value falls in.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace spkb::dev {

template <int N>
struct Dual {
    float v;
    float d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dconst(float v) {
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = 0.0f;
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> dvar(float v, int i) {
    Dual<N> r = dconst<N>(v);
    r.d[i] = 1.0f;
    return r;
}

// With an even number of tangents the tangent arithmetic runs on packed f32x2 operations, tangents i and
// i + 1 in the two halves (half the instructions; each half is the same IEEE operation as the scalar form).
template <int N>
__device__ __forceinline__ float2 dpair(const Dual<N>& a, int i) {
    return make_float2(a.d[i], a.d[i + 1]);
}
template <int N>
__device__ __forceinline__ void dset(Dual<N>& r, int i, float2 v) {
    r.d[i] = v.x;
    r.d[i + 1] = v.y;
}
__device__ __forceinline__ float2 dsplat(float v) { return make_float2(v, v); }

// r = a + b, a - b, a * b, a / b
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
    if constexpr (N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2) dset(r, i, __fadd2_rn(dpair(a, i), dpair(b, i)));
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    }
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
    if constexpr (N % 2 == 0) {
        // a - b as fma(b, -1, a): the product is exact, so one rounding as in the scalar subtraction
#pragma unroll
        for (int i = 0; i < N; i += 2) dset(r, i, __ffma2_rn(dpair(b, i), dsplat(-1.0f), dpair(a, i)));
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    }
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
    if constexpr (N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2)
            dset(r, i, __ffma2_rn(dpair(a, i), dsplat(b.v), __fmul2_rn(dsplat(a.v), dpair(b, i))));
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    }
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const float ib = 1.0f / b.v;
    if constexpr (N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2)
            dset(r, i, __fmul2_rn(__ffma2_rn(dpair(b, i), dsplat(-r.v), dpair(a, i)), dsplat(ib)));
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    }
    return r;
}
// with a constant
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, float b) {
    Dual<N> r = a;
    r.v = a.v + b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(float b, const Dual<N>& a) {
    return a + b;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, float b) {
    Dual<N> r = a;
    r.v = a.v - b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(float b, const Dual<N>& a) {
    Dual<N> r;
    r.v = b - a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, float b) {
    Dual<N> r;
    r.v = a.v * b;
    if constexpr (N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2) dset(r, i, __fmul2_rn(dpair(a, i), dsplat(b)));
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    }
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(float b, const Dual<N>& a) {
    return a * b;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, float b) {
    Dual<N> r;
    r.v = a.v / b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(float a, const Dual<N>& b) {
    return dconst<N>(a) / b;
}

// f(a) with f'(a) given
template <int N>
__device__ __forceinline__ Dual<N> dchain(const Dual<N>& a, float fv, float fd) {
    Dual<N> r;
    r.v = fv;
    if constexpr (N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2) dset(r, i, __fmul2_rn(dsplat(fd), dpair(a, i)));
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = fd * a.d[i];
    }
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> dexp(const Dual<N>& a) {
    const float e = expf(a.v);
    return dchain(a, e, e);
}
template <int N>
__device__ __forceinline__ Dual<N> dlog(const Dual<N>& a) {
    return dchain(a, logf(a.v), 1.0f / a.v);
}
template <int N>
__device__ __forceinline__ Dual<N> dlog10(const Dual<N>& a) {
    return dchain(a, log10f(a.v), 0.43429448190325182f / a.v);
}
// 10^a
template <int N>
__device__ __forceinline__ Dual<N> dexp10(const Dual<N>& a) {
    const float e = exp10f(a.v);
    return dchain(a, e, 2.30258509299404568f * e);
}
template <int N>
__device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
    const float s = sqrtf(a.v);
    return dchain(a, s, s > 0.0f ? 0.5f / s : 0.0f);
}
// |a|^p for p > 0, the tangent 0 at a = 0
template <int N>
__device__ __forceinline__ Dual<N> dpow(const Dual<N>& a, float p) {
    const float v = powf(a.v, p);
    return dchain(a, v, a.v > 0.0f ? p * v / a.v : 0.0f);
}
template <int N>
__device__ __forceinline__ Dual<N> dfabs(const Dual<N>& a) {
    return a.v < 0.0f ? -a : a;
}
template <int N>
__device__ __forceinline__ Dual<N> dfmax(const Dual<N>& a, float b) {
    return a.v >= b ? a : dconst<N>(b);
}
template <int N>
__device__ __forceinline__ Dual<N> dfmin(const Dual<N>& a, float b) {
    return a.v <= b ? a : dconst<N>(b);
}
template <int N>
__device__ __forceinline__ Dual<N> dclamp(const Dual<N>& a, float lo, float hi) {
    return dfmin(dfmax(a, lo), hi);
}
template <int N>
__device__ __forceinline__ Dual<N> dsin(const Dual<N>& a) {
    float s, c;
    sincosf(a.v, &s, &c);
    return dchain(a, s, c);
}
template <int N>
__device__ __forceinline__ Dual<N> dcos(const Dual<N>& a) {
    float s, c;
    sincosf(a.v, &s, &c);
    return dchain(a, c, -s);
}
template <int N>
__device__ __forceinline__ Dual<N> datan2(const Dual<N>& y, const Dual<N>& x) {
    Dual<N> r;
    r.v = atan2f(y.v, x.v);
    const float q = x.v * x.v + y.v * y.v;
    const float iq = q > 0.0f ? 1.0f / q : 0.0f;
    if constexpr (N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2)
            dset(r, i, __fmul2_rn(__ffma2_rn(dpair(x, i), dsplat(-y.v), __fmul2_rn(dsplat(x.v), dpair(y, i))),
                                  dsplat(iq)));
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) * iq;
    }
    return r;
}
// sign(a) as a constant
template <int N>
__device__ __forceinline__ float dsgn(const Dual<N>& a) {
    return a.v > 0.0f ? 1.0f : (a.v < 0.0f ? -1.0f : 0.0f);
}

// a 3 x 3 matrix (row-major, constant) times a vector of duals, in the reference's bracketing
template <int N>
__device__ __forceinline__ void dmat(const float* m, const Dual<N>& x, const Dual<N>& y, const Dual<N>& z, Dual<N>& a,
                                     Dual<N>& b, Dual<N>& c) {
    a = (m[0] * x + m[1] * y) + m[2] * z;
    b = (m[3] * x + m[4] * y) + m[5] * z;
    c = (m[6] * x + m[7] * y) + m[8] * z;
}

}  // namespace spkb::dev
