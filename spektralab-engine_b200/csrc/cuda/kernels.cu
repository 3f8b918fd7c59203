// sm_100a kernels of the render path (first generation: one pass per stage, fused where the reference
// stores and reloads an intermediate plane with no change of value).
//
// Numerics follow the reference kernels (kernels/film.metal, print.metal, fx_blur.metal,
// fx_grain.metal): binary32 arithmetic in the same bracketing; recursive-filter state in binary64
// (the reference keeps it in double-float on its GPU and in double on its host copy); the grain
// sampler from grain_sampler.h, which the host checker compiles too.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <mutex>

#include "../grain_sampler.h"
#include "../kernel_args.h"
#include "encode.cuh"
#include "launch.hpp"
#include "lookup.cuh"

namespace spkb::dev {

namespace {

__host__ __device__ inline uint32_t div_up(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------------------------------
// expose: reference kernels/film.metal:50-99 (Mitchell-Netravali B = C = 1/3) and :189-227.

__device__ __forceinline__ float mitchell(float u) {
    const float a = fabsf(u);
    if (a < 1.0f) return (1.0f / 6.0f) * (7.0f * a * a * a - 12.0f * a * a + 16.0f / 3.0f);
    if (a < 2.0f) return (1.0f / 6.0f) * ((-7.0f / 3.0f) * a * a * a + 12.0f * a * a - 20.0f * a + 32.0f / 3.0f);
    return 0.0f;
}

__device__ __forceinline__ void mitchell_axis(float t, uint32_t L, int* idx, float* w) {
    const float last = float(L - 1);
    float u = t * last;
    int base;
    float frac;
    if (u <= 0.0f) u = 0.0f;
    if (u >= last) {
        base = int(L) - 2;
        frac = 1.0f;
    } else {
        base = int(floorf(u));
        frac = u - float(base);
    }
    const int n = int(L);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int i = base - 1 + k;
        if (i < 0) i = -i;
        if (i >= n) i = 2 * (n - 1) - i;
        idx[k] = i;
    }
    w[0] = mitchell(frac + 1.0f);
    w[1] = mitchell(frac);
    w[2] = mitchell(frac - 1.0f);
    w[3] = mitchell(frac - 2.0f);
}

__global__ void k_expose(const float* __restrict__ rgb, float* __restrict__ hout, const float4* __restrict__ table,
                         const __grid_constant__ ExposeArgs q) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= q.n) return;
    float r = rgb[3 * size_t(gid)], g = rgb[3 * size_t(gid) + 1], b = rgb[3 * size_t(gid) + 2];
    if (q.apply_ae) {  // the auto-exposure scale pass (reference src/film/develop.cpp:132-140), one rounding each
        r = __fmul_rn(r, q.ae_gain);
        g = __fmul_rn(g, q.ae_gain);
        b = __fmul_rn(b, q.ae_gain);
    }
    const float X = (q.a[0] * r + q.a[1] * g) + q.a[2] * b;
    const float Y = (q.a[3] * r + q.a[4] * g) + q.a[5] * b;
    const float Z = (q.a[6] * r + q.a[7] * g) + q.a[8] * b;
    const float bs = (X + Y) + Z;
    const float d = bs > 1e-10f ? bs : 1e-10f;
    const float x = X / d, y = Y / d, o = 1.0f - x;
    const float t0 = fminf(fmaxf(o * o, 0.0f), 1.0f);
    const float t1 = fminf(fmaxf(y / (o > 1e-10f ? o : 1e-10f), 0.0f), 1.0f);
    const float bp = isnan(bs) ? 0.0f : bs;
    int ia[4], ib[4];
    float wa[4], wb[4];
    mitchell_axis(t0, q.L, ia, wa);
    mitchell_axis(t1, q.L, ib, wb);
    float s = 0.0f, a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float w = wa[i] * wb[j];
            const float4 t = __ldg(table + (size_t(ia[i]) * q.L + size_t(ib[j])));
            s += w;
            a0 += w * t.x;
            a1 += w * t.y;
            a2 += w * t.z;
        }
    }
    if (s != 0.0f) {
        a0 = a0 / s;
        a1 = a1 / s;
        a2 = a2 / s;
    }
    float h0 = bp * a0, h1 = bp * a1, h2 = bp * a2;
    if (q.apply_gain) {
        h0 = h0 * q.gain;
        h1 = h1 * q.gain;
        h2 = h2 * q.gain;
    }
    hout[3 * size_t(gid)] = h0;
    hout[3 * size_t(gid) + 1] = h1;
    hout[3 * size_t(gid) + 2] = h2;
}

// The same pass over a table of 4 x 4 patches. Patch (ba, bb) holds the sixteen texels the bicubic reads
// when the pixel's base indices are (ba, bb) -- row reflect(ba - 1 + i), column reflect(bb - 1 + j) -- as
// RGB triples in the loop order (i outer, j inner): 48 floats, 192 bytes, fetched with six 32-byte loads
// instead of sixteen 16-byte gathers, so a warp's random lookups take about a third of the L1 wavefronts.
// The arithmetic is k_expose's, operation for operation. Four pixels per thread, read and written as three
// 16-byte vectors each.

__device__ __forceinline__ void mitchell_base(float t, uint32_t L, int& base, float w[4]) {
    const float last = float(L - 1);
    float u = t * last;
    float frac;
    if (u <= 0.0f) u = 0.0f;
    if (u >= last) {
        base = int(L) - 2;
        frac = 1.0f;
    } else {
        base = int(floorf(u));
        frac = u - float(base);
    }
    w[0] = mitchell(frac + 1.0f);
    w[1] = mitchell(frac);
    w[2] = mitchell(frac - 1.0f);
    w[3] = mitchell(frac - 2.0f);
}

__device__ __forceinline__ void ld32(const float* p, float* r) {
    asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
                 : "l"(p));
}

__device__ __forceinline__ void expose_pixel(const ExposeArgs& q, const float* __restrict__ patches, float r, float g,
                                             float b, float* h) {
    if (q.apply_ae) {
        r = __fmul_rn(r, q.ae_gain);
        g = __fmul_rn(g, q.ae_gain);
        b = __fmul_rn(b, q.ae_gain);
    }
    const float X = (q.a[0] * r + q.a[1] * g) + q.a[2] * b;
    const float Y = (q.a[3] * r + q.a[4] * g) + q.a[5] * b;
    const float Z = (q.a[6] * r + q.a[7] * g) + q.a[8] * b;
    const float bs = (X + Y) + Z;
    const float d = bs > 1e-10f ? bs : 1e-10f;
    const float x = X / d, y = Y / d, o = 1.0f - x;
    const float t0 = fminf(fmaxf(o * o, 0.0f), 1.0f);
    const float t1 = fminf(fmaxf(y / (o > 1e-10f ? o : 1e-10f), 0.0f), 1.0f);
    const float bp = isnan(bs) ? 0.0f : bs;
    int ba, bb;
    float wa[4], wb[4];
    mitchell_base(t0, q.L, ba, wa);
    mitchell_base(t1, q.L, bb, wb);
    const float* pt = patches + (size_t(ba) * (q.L - 1) + size_t(bb)) * kPatchFloats;
    float t[kPatchFloats];
#pragma unroll
    for (int k = 0; k < 6; ++k) ld32(pt + 8 * k, t + 8 * k);
    float s = 0.0f, a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float w = wa[i] * wb[j];
            const float* tx = t + 3 * (4 * i + j);
            s += w;
            a0 += w * tx[0];
            a1 += w * tx[1];
            a2 += w * tx[2];
        }
    }
    if (s != 0.0f) {
        a0 = a0 / s;
        a1 = a1 / s;
        a2 = a2 / s;
    }
    float h0 = bp * a0, h1 = bp * a1, h2 = bp * a2;
    if (q.apply_gain) {
        h0 = h0 * q.gain;
        h1 = h1 * q.gain;
        h2 = h2 * q.gain;
    }
    h[0] = h0;
    h[1] = h1;
    h[2] = h2;
}

#ifndef SPKB_EXPOSE_THREADS
#define SPKB_EXPOSE_THREADS 128
#endif
constexpr uint32_t kExposeThreads = SPKB_EXPOSE_THREADS;

__global__ void __launch_bounds__(kExposeThreads) k_expose_patch(const float* __restrict__ rgb, float* __restrict__ hout,
                                                                 const float* __restrict__ patches,
                                                                 const __grid_constant__ ExposeArgs q) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t p0 = 4 * t;
    if (p0 >= q.n) return;
    if (p0 + 4 <= q.n) {
        const float4* src = reinterpret_cast<const float4*>(rgb) + 3 * size_t(t);
        const float4 v0 = __ldcs(src), v1 = __ldcs(src + 1), v2 = __ldcs(src + 2);
        const float in[12] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w, v2.x, v2.y, v2.z, v2.w};
        float out[12];
#pragma unroll
        for (int k = 0; k < 4; ++k) expose_pixel(q, patches, in[3 * k], in[3 * k + 1], in[3 * k + 2], out + 3 * k);
        float4* dst = reinterpret_cast<float4*>(hout) + 3 * size_t(t);
        dst[0] = make_float4(out[0], out[1], out[2], out[3]);
        dst[1] = make_float4(out[4], out[5], out[6], out[7]);
        dst[2] = make_float4(out[8], out[9], out[10], out[11]);
    } else {
        for (uint32_t p = p0; p < q.n; ++p)
            expose_pixel(q, patches, rgb[3 * size_t(p)], rgb[3 * size_t(p) + 1], rgb[3 * size_t(p) + 2],
                         hout + 3 * size_t(p));
    }
}

// ---------------------------------------------------------------------------------------------------
// FIR: reference kernels/fx_blur.metal:20-78: taps -r..r ascending, float accumulator from 0,
// half-sample symmetric reflection at the edges.

__device__ __forceinline__ int reflect_index(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * n;
    int m = i % period;
    if (m < 0) m += period;
    return m < n ? m : period - 1 - m;
}

__global__ void k_fir_v(const float* __restrict__ in, float* __restrict__ out, uint32_t w, uint32_t h,
                        const __grid_constant__ FirTaps t) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int r = t.r;
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    for (int i = -r; i <= r; ++i) {
        const int yy = reflect_index(int(y) + i, int(h));
        const float* p = in + 3 * (size_t(yy) * w + x);
        const int k = i + r;
        a0 += t.taps[0][k] * p[0];
        a1 += t.taps[1][k] * p[1];
        a2 += t.taps[2][k] * p[2];
    }
    float* o = out + 3 * (size_t(y) * w + x);
    o[0] = a0;
    o[1] = a1;
    o[2] = a2;
}

__global__ void k_fir_h(const float* __restrict__ in, float* out, const float* acc, uint32_t w, uint32_t h,
                        const __grid_constant__ FirTaps t, int mode, float w0, float w1, float w2) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int r = t.r;
    const float* row = in + 3 * size_t(y) * w;
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    for (int i = -r; i <= r; ++i) {
        const int xx = reflect_index(int(x) + i, int(w));
        const float* p = row + 3 * xx;
        const int k = i + r;
        a0 += t.taps[0][k] * p[0];
        a1 += t.taps[1][k] * p[1];
        a2 += t.taps[2][k] * p[2];
    }
    const size_t o = 3 * (size_t(y) * w + x);
    if (mode == ACC_NONE) {
        out[o] = a0;
        out[o + 1] = a1;
        out[o + 2] = a2;
    } else if (mode == ACC_ZERO) {
        out[o] = 0.0f + w0 * a0;
        out[o + 1] = 0.0f + w1 * a1;
        out[o + 2] = 0.0f + w2 * a2;
    } else {
        const float c0 = acc[o], c1 = acc[o + 1], c2 = acc[o + 2];
        out[o] = c0 + w0 * a0;
        out[o + 1] = c1 + w1 * a1;
        out[o + 2] = c2 + w2 * a2;
    }
}

// ---------------------------------------------------------------------------------------------------
// Recursive Gaussian (Young-van Vliet, third order): reference kernels/fx_blur.metal:125-204.
//   forward:  w[-1..-3] = x[0];  w[i] = B x[i] + B1 w[i-1] + B2 w[i-2] + B3 w[i-3];  u[i] = float(w[i])
//   backward: y[n..n+2] = u[n-1]; y[i] = B u[i] + B1 y[i+1] + B2 y[i+2] + B3 y[i+3]
// State in binary64; x, u and y stored as binary32.

__device__ __forceinline__ void iir_line(const float* src, float* work, float* dst, const float* acc, size_t base,
                                         size_t stride, uint32_t n, const IirCoefs& q, int c, int mode,
                                         float wgt) {
    const double B = q.B[c], B1 = q.B1[c], B2 = q.B2[c], B3 = q.B3[c];
    double w1 = double(src[base]), w2 = w1, w3 = w1;
    for (uint32_t i = 0; i < n; ++i) {
        const size_t o = base + i * stride;
        const double t = ((B * double(src[o]) + B1 * w1) + B2 * w2) + B3 * w3;
        w3 = w2;
        w2 = w1;
        w1 = t;
        work[o] = float(t);
    }
    double y1 = double(work[base + size_t(n - 1) * stride]), y2 = y1, y3 = y1;
    for (uint32_t k = n; k-- > 0;) {
        const size_t o = base + k * stride;
        const double t = ((B * double(work[o]) + B1 * y1) + B2 * y2) + B3 * y3;
        y3 = y2;
        y2 = y1;
        y1 = t;
        const float y = float(t);
        if (mode == ACC_NONE) dst[o] = y;
        else if (mode == ACC_ZERO) dst[o] = 0.0f + wgt * y;
        else dst[o] = acc[o] + wgt * y;
    }
}

// The same line with its tangent along sigma (forward mode): the coefficients' derivatives dq (the same
// layout as q) and the input's tangent src_dot (nullptr: zero) give the output's tangent
//   forward:  w'[i] = dB x[i] + B x'[i] + sum_j (dB_j w[i-j] + B_j w'[i-j]), w'[-1..-3] = x'[0]
//   backward: y'[i] = dB u[i] + B u'[i] + sum_j (dB_j y[i+j] + B_j y'[i+j]), y'[n..n+2] = u'[n-1]
// with u = the forward pass rounded to binary32 (its tangent is not rounded). Work planes: the forward
// pass's value and tangent.
__device__ __forceinline__ void iir_line_tangent(const float* __restrict__ src, const float* __restrict__ src_dot,
                                                 float* __restrict__ work, float* __restrict__ work_dot,
                                                 float* __restrict__ dst, float* __restrict__ dst_dot, size_t base,
                                                 size_t stride, uint32_t n, const IirCoefs& q, const IirCoefs& dq,
                                                 int c) {
    // the line's samples go in chunks of kTanChunk: a chunk's loads are issued together, ahead of its
    // recurrence steps, so that a step waits on the previous step and not on memory
    constexpr uint32_t kTanChunk = 8;
    const double B = q.B[c], B1 = q.B1[c], B2 = q.B2[c], B3 = q.B3[c];
    const double dB = dq.B[c], dB1 = dq.B1[c], dB2 = dq.B2[c], dB3 = dq.B3[c];
    double w1 = double(src[base]), w2 = w1, w3 = w1;
    double t1 = src_dot ? double(src_dot[base]) : 0.0, t2 = t1, t3 = t1;
    for (uint32_t i0 = 0; i0 < n; i0 += kTanChunk) {
        float xs[kTanChunk], xds[kTanChunk];
#pragma unroll
        for (uint32_t j = 0; j < kTanChunk; ++j) {
            const size_t o = base + size_t(i0 + j) * stride;
            xs[j] = i0 + j < n ? src[o] : 0.0f;
            xds[j] = i0 + j < n && src_dot ? src_dot[o] : 0.0f;
        }
#pragma unroll
        for (uint32_t j = 0; j < kTanChunk; ++j) {
            if (i0 + j >= n) break;
            const size_t o = base + size_t(i0 + j) * stride;
            const double x = double(xs[j]), xd = double(xds[j]);
            // the newest state enters last: one multiply-add latency per sample on each recurrence
            const double v = fma(B1, w1, fma(B2, w2, fma(B3, w3, B * x)));
            const double vd = fma(B1, t1, fma(dB1, w1, fma(B2, t2, fma(dB2, w2, fma(B3, t3, fma(dB3, w3, fma(B, xd, dB * x)))))));
            w3 = w2;
            w2 = w1;
            w1 = v;
            t3 = t2;
            t2 = t1;
            t1 = vd;
            work[o] = float(v);
            work_dot[o] = float(vd);
        }
    }
    const size_t last = base + size_t(n - 1) * stride;
    double y1 = double(work[last]), y2 = y1, y3 = y1;
    double s1 = double(work_dot[last]), s2 = s1, s3 = s1;
    for (uint32_t k0 = n; k0 > 0;) {
        const uint32_t m = k0 < kTanChunk ? k0 : kTanChunk;  // samples k0 - 1 down to k0 - m
        float us[kTanChunk], uds[kTanChunk];
#pragma unroll
        for (uint32_t j = 0; j < kTanChunk; ++j) {
            const size_t o = base + size_t(k0 - 1 - (j < m ? j : 0)) * stride;
            us[j] = work[o];
            uds[j] = work_dot[o];
        }
#pragma unroll
        for (uint32_t j = 0; j < kTanChunk; ++j) {
            if (j >= m) break;
            const size_t o = base + size_t(k0 - 1 - j) * stride;
            const double u = double(us[j]), ud = double(uds[j]);
            const double v = fma(B1, y1, fma(B2, y2, fma(B3, y3, B * u)));
            const double vd = fma(B1, s1, fma(dB1, y1, fma(B2, s2, fma(dB2, y2, fma(B3, s3, fma(dB3, y3, fma(B, ud, dB * u)))))));
            y3 = y2;
            y2 = y1;
            y1 = v;
            s3 = s2;
            s2 = s1;
            s1 = vd;
            dst[o] = float(v);
            dst_dot[o] = float(vd);
        }
        k0 -= m;
    }
}

// The same tangent with the lines staged in shared memory and each line cut into kTanSegs segments of L
// samples, a thread per (line, segment). A CTA takes `px` rows (3 px lines, vertical = 0) or a strip of
// `px` pixel columns (3 px lines, vertical = 1); the whole CTA loads and stores them in the frame's order.
// Line j, sample i at [i * nl + j]. The value and its tangent form one linear recurrence on the state
// (w1, w2, w3, t1, t2, t3) (the last three values and tangents), so a segment is solved block-parallel as
// the blur itself is: every segment runs from a zero state (the first from the line's edge state) and
// keeps its end state e_s; one thread per line chains the true entry states, S_{s+1} = A^L S_s + e_s, with
// A^L the homogeneous L-step map (TangentMaps, binary64, formed on the host); every segment then reruns
// from its true entry state and stores float(value) and float(tangent) in place. The backward direction
// cuts its segments from the line's end. The state is binary64 throughout.
constexpr uint32_t kTanSegs = 8;
struct TangentMaps {
    double AL[3][36];  // per channel, row-major over (w1, w2, w3, t1, t2, t3)
    uint32_t L;        // segment length
};

struct TanState {
    double w1, w2, w3, t1, t2, t3;
};

// one step of the recurrence on the sample at smem offset o (x and its tangent), the newest state last in
// each multiply-add chain; writes float(value), float(tangent) back when `store`
__device__ __forceinline__ void tan_step(TanState& st, const double* k, float* val, float* dot, size_t o, bool store) {
    const double x = double(val[o]), xd = double(dot[o]);
    const double v = fma(k[1], st.w1, fma(k[2], st.w2, fma(k[3], st.w3, k[0] * x)));
    const double vd = fma(k[1], st.t1, fma(k[5], st.w1, fma(k[2], st.t2, fma(k[6], st.w2,
                      fma(k[3], st.t3, fma(k[7], st.w3, fma(k[0], xd, k[4] * x)))))));
    st.w3 = st.w2;
    st.w2 = st.w1;
    st.w1 = v;
    st.t3 = st.t2;
    st.t2 = st.t1;
    st.t1 = vd;
    if (store) {
        val[o] = float(v);
        dot[o] = float(vd);
    }
}

__global__ void k_iir_tangent_seg(const float* __restrict__ in, const float* __restrict__ in_dot,
                                  float* __restrict__ out, float* __restrict__ out_dot, uint32_t w, uint32_t h,
                                  int vertical, uint32_t px, const __grid_constant__ IirCoefs q,
                                  const __grid_constant__ IirCoefs dq, const __grid_constant__ TangentMaps maps) {
    extern __shared__ __align__(16) unsigned char tsm_raw[];
    const uint32_t n = vertical ? h : w;
    const uint32_t z0 = blockIdx.x * px;                    // the first pixel column, or row
    const uint32_t npx = min(px, (vertical ? w : h) - z0);  // columns (rows) in this strip
    const uint32_t nl = 3 * px;                              // the strip's line pitch
    const uint32_t nv = 3 * npx;                             // valid lines
    double* carry = reinterpret_cast<double*>(tsm_raw);      // [line][segment][6]
    float* val = reinterpret_cast<float*>(carry + size_t(nl) * kTanSegs * 6);
    float* dot = val + size_t(n) * nl;
    const uint32_t span = vertical ? nv : 3 * n;  // contiguous floats per strip row
    const uint32_t total = vertical ? n * nv : npx * 3 * n;
#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
        const uint32_t r = e / span, f = e - r * span;
        const size_t g = vertical ? (size_t(r) * w + z0) * 3 + f : (size_t(z0 + r) * w) * 3 + f;
        const uint32_t i = vertical ? r : f / 3, j = vertical ? f : 3 * r + f % 3;
        val[size_t(i) * nl + j] = in[g];
        dot[size_t(i) * nl + j] = in_dot ? in_dot[g] : 0.0f;
    }
    __syncthreads();

    const uint32_t line = threadIdx.x / kTanSegs, seg = threadIdx.x % kTanSegs;
    const int c = int(line % 3u);
    const bool active = line < nv && ((q.mask >> c) & 1u) != 0u;
    const double k[8] = {q.B[c], q.B1[c], q.B2[c], q.B3[c], dq.B[c], dq.B1[c], dq.B2[c], dq.B3[c]};
    const uint32_t L = maps.L;
    double* cs = carry + (size_t(line) * kTanSegs + seg) * 6;
    for (int dir = 0; dir < 2; ++dir) {
        // this segment's samples: forward [a, b) ascending; backward [a, b) descending, cut from the end
        uint32_t a, b;
        if (dir == 0) {
            a = min(n, seg * L);
            b = min(n, a + L);
        } else {
            b = n > seg * L ? n - seg * L : 0u;
            a = b > L ? b - L : 0u;
        }
        // the line's edge state: x[0] (forward) or the forward result u[n-1] (backward)
        TanState edge{};
        if (active) {
            const size_t o0 = size_t(dir == 0 ? 0u : n - 1u) * nl + line;
            const double e0 = double(val[o0]), d0 = double(dot[o0]);
            edge = TanState{e0, e0, e0, d0, d0, d0};
        }
        // pass 1: zero-state run (the first segment from the edge state), its end state kept
        if (active && a < b) {
            TanState st = seg == 0 ? edge : TanState{};
            if (dir == 0) {
                for (uint32_t i = a; i < b; ++i) tan_step(st, k, val, dot, size_t(i) * nl + line, false);
            } else {
                for (uint32_t i = b; i-- > a;) tan_step(st, k, val, dot, size_t(i) * nl + line, false);
            }
            cs[0] = st.w1;
            cs[1] = st.w2;
            cs[2] = st.w3;
            cs[3] = st.t1;
            cs[4] = st.t2;
            cs[5] = st.t3;
        }
        __syncthreads();
        // the true entry states, one thread per line: segment s + 1 enters with A^L S_s + e_s (segment 0's
        // end state is already true); a segment's slot takes its entry state
        if (active && seg == 0) {
            double S[6];
            double* c0 = carry + size_t(line) * kTanSegs * 6;
            for (int m = 0; m < 6; ++m) S[m] = c0[m];
            for (uint32_t sg = 1; sg < kTanSegs && sg * L < n; ++sg) {
                double* cg = c0 + sg * 6;
                double e[6];
                for (int m = 0; m < 6; ++m) {
                    e[m] = cg[m];
                    cg[m] = S[m];
                }
                const double* A = maps.AL[c];
                double T[6];
                for (int r = 0; r < 6; ++r) {
                    double acc = e[r];
                    for (int m = 0; m < 6; ++m) acc = fma(A[r * 6 + m], S[m], acc);
                    T[r] = acc;
                }
                for (int m = 0; m < 6; ++m) S[m] = T[m];
            }
        }
        __syncthreads();
        // pass 2: every segment from its true entry state, storing
        if (active && a < b) {
            TanState st = seg == 0 ? edge : TanState{cs[0], cs[1], cs[2], cs[3], cs[4], cs[5]};
            if (dir == 0) {
                for (uint32_t i = a; i < b; ++i) tan_step(st, k, val, dot, size_t(i) * nl + line, true);
            } else {
                for (uint32_t i = b; i-- > a;) tan_step(st, k, val, dot, size_t(i) * nl + line, true);
            }
        }
        __syncthreads();
    }
#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
        const uint32_t r = e / span, f = e - r * span;
        const size_t g = vertical ? (size_t(r) * w + z0) * 3 + f : (size_t(z0 + r) * w) * 3 + f;
        const uint32_t i = vertical ? r : f / 3, j = vertical ? f : 3 * r + f % 3;
        out[g] = val[size_t(i) * nl + j];
        out_dot[g] = dot[size_t(i) * nl + j];
    }
}

// the blur's tangent along sigma, one thread per line: rows (vertical = 0) or columns (vertical = 1); a
// channel outside q.mask passes its value and tangent through
__global__ void k_iir_tangent(const float* __restrict__ in, const float* in_dot, float* work, float* work_dot,
                              float* out, float* out_dot, uint32_t w, uint32_t h, int vertical,
                              const __grid_constant__ IirCoefs q, const __grid_constant__ IirCoefs dq) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lines = vertical ? 3u * w : 3u * h;
    if (t >= lines) return;
    const uint32_t c = t % 3u;
    const size_t base = vertical ? size_t(t) : 3 * size_t(t / 3u) * w + c;
    const size_t stride = vertical ? 3 * size_t(w) : 3;
    const uint32_t n = vertical ? h : w;
    if (((q.mask >> c) & 1u) == 0u) {
        for (uint32_t i = 0; i < n; ++i) {
            const size_t o = base + i * stride;
            out[o] = in[o];
            out_dot[o] = in_dot ? in_dot[o] : 0.0f;
        }
        return;
    }
    iir_line_tangent(in, in_dot, work, work_dot, out, out_dot, base, stride, n, q, dq, int(c));
}

__global__ void k_iir_h(const float* __restrict__ in, float* out, uint32_t w, uint32_t h,
                        const __grid_constant__ IirCoefs q) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3u * h) return;
    const uint32_t y = t / 3u, c = t % 3u;
    const size_t base = 3 * size_t(y) * w + c;
    if (((q.mask >> c) & 1u) == 0u) {
        for (uint32_t x = 0; x < w; ++x) out[base + 3 * size_t(x)] = in[base + 3 * size_t(x)];
        return;
    }
    iir_line(in, out, out, out, base, 3, w, q, int(c), ACC_NONE, 1.0f);
}

__global__ void k_iir_v(float* work, float* out, const float* acc, uint32_t w, uint32_t h,
                        const __grid_constant__ IirCoefs q, int mode, float w0, float w1, float w2) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3u * w) return;
    const uint32_t c = t % 3u;
    const size_t stride = 3 * size_t(w);
    if (((q.mask >> c) & 1u) == 0u) {
        for (uint32_t y = 0; y < h; ++y) out[t + y * stride] = work[t + y * stride];
        return;
    }
    const float wgt = c == 0 ? w0 : (c == 1 ? w1 : w2);
    iir_line(work, work, out, acc, t, stride, h, q, int(c), mode, wgt);
}

__global__ void k_lincomb(const float* x, const float* y, float* out, size_t n, float a0, float a1, float a2,
                          float b0, float b1, float b2) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float a[3] = {a0, a1, a2}, b[3] = {b0, b1, b2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const size_t o = 3 * i + c;
        const float yv = y ? y[o] : 0.0f;
        out[o] = a[c] * x[o] + b[c] * yv;
    }
}

__global__ void k_copy(const float* __restrict__ x, float* __restrict__ out, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = x[i];
}

// ---------------------------------------------------------------------------------------------------
// develop: log10 exposure (film.metal:242-246), density curves (:84-101, :249-261), grain draw
// (fx_grain.metal:39-97, SUM and SIMPLE modes).

__device__ __forceinline__ float curve_lookup(const float* __restrict__ x, const float* __restrict__ inv,
                                              const float* __restrict__ y, uint32_t K, const AxisGrid& g, float v) {
    if (v <= __ldg(x)) return __ldg(y);
    if (v >= __ldg(x + K - 1)) return __ldg(y + K - 1);
    const uint32_t l = axis_index(x, 1, K, g, v);
    const float t = (v - __ldg(x + l)) * __ldg(inv + l);
    const float y0 = __ldg(y + l);
    return y0 + t * (__ldg(y + l + 1) - y0);
}

// the three sub-layer densities of channel c at density v (reference fx_grain.metal:60-75)
__device__ __forceinline__ void layer_densities(const DevelopArgs& q, uint32_t c, float v, float dl[3]) {
    const uint32_t K = q.gK;
    if (v <= __ldg(q.axis + c)) {
        for (uint32_t l = 0; l < 3u; ++l) dl[l] = __ldg(q.layers + l * 3u + c);
    } else if (v >= __ldg(q.axis + 3u * (K - 1u) + c)) {
        for (uint32_t l = 0; l < 3u; ++l) dl[l] = __ldg(q.layers + ((K - 1u) * 3u + l) * 3u + c);
    } else {
        // a NaN v gives j = 0, in bounds, and NaN densities
        const uint32_t j = axis_index(q.axis + c, 3u, K, q.ggrid[c], v);
        const float t = (v - __ldg(q.axis + 3u * j + c)) * __ldg(q.ginv + 3u * j + c);
        for (uint32_t l = 0; l < 3u; ++l) {
            const float y0 = __ldg(q.layers + (j * 3u + l) * 3u + c);
            const float y1 = __ldg(q.layers + ((j + 1u) * 3u + l) * 3u + c);
            dl[l] = y0 + t * (y1 - y0);
        }
    }
}

// spk_sublayer_draw (grain_sampler.h) with the count kept for the test hook: the same operations.
__device__ __forceinline__ float grain_draw(float d, float D, float n, float u, uint32_t pixel, uint32_t stream,
                                            uint32_t seed, float* count_slot) {
    float sat;
    const float lam = spk_sublayer_lambda(d, D, n, u, &sat);
    const float k = spk_poisson(lam, pixel, stream, seed);
    if (count_slot) *count_slot = k;
    return SPK_MUL(k, SPK_MUL(SPK_DIV(D, n), sat));
}

// DIR couplers' source (reference kernels/film.metal:242-276): L = log10(max(H, 0) + 1e-10), D = the curve at
// L, s_c = positive ? dmax_c - D_c : D_c, chi_m = (s_0 M[0][m] + s_1 M[1][m]) + s_2 M[2][m], each operation
// rounded as written
__global__ void k_coupler_source(const float* __restrict__ exposure, float* __restrict__ chi,
                                 const __grid_constant__ CouplerArgs q) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    float sv[3];
#pragma unroll
    for (uint32_t c = 0; c < 3; ++c) {
        const float L = log10f(fmaxf(exposure[3 * size_t(i) + c], 0.0f) + 1e-10f);
        const float D = curve_lookup(q.cx, q.cinv, q.cy + size_t(c) * q.K, q.K, q.cgrid, L);
        sv[c] = q.positive ? __fsub_rn(q.dmax[c], D) : D;
    }
#pragma unroll
    for (uint32_t m = 0; m < 3; ++m)
        chi[3 * size_t(i) + m] = __fadd_rn(__fadd_rn(__fmul_rn(sv[0], q.m[m]), __fmul_rn(sv[1], q.m[3 + m])),
                                           __fmul_rn(sv[2], q.m[6 + m]));
}

__global__ void k_develop(const float* __restrict__ exposure, float* __restrict__ out, uint32_t w, uint32_t h,
                          const __grid_constant__ DevelopArgs q) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const uint32_t pixel = y * q.width + x;
    const size_t o = 3 * (size_t(y) * w + x);
    for (uint32_t c = 0; c < 3; ++c) {
        float L = log10f(fmaxf(exposure[o + c], 0.0f) + 1e-10f);
        if (q.chi) L = __fsub_rn(L, q.chi[o + c]);  // DIR couplers: the corrected log exposure, the y0 curve
        const float D = curve_lookup(q.cx, q.cinv, q.cy + size_t(c) * q.K, q.K, q.cgrid, L);
        if (!q.grain) {
            out[o + c] = D;
            continue;
        }
        if (q.mode == 2) {  // SIMPLE
            const float d = D + q.dmin_c[c];
            float G = 0.0f;
            for (uint32_t l = 0; l < q.n_sub; ++l)
                G = G + grain_draw(d, q.sat_d[c], q.count[c], q.uniformity[c], pixel, SPK_STREAM_GRAIN(c, l), q.seed,
                                   q.counts_out && l < 3 ? q.counts_out + size_t(pixel) * 9 + c * 3 + l : nullptr);
            out[o + c] = G * q.inv_n_sub + (-q.dmin_c[c]);
            continue;
        }
        const float v = q.positive ? -D : D;
        float dl[3];
        layer_densities(q, c, v, dl);
        float val[3];
        for (uint32_t l = 0; l < 3u; ++l) {
            const uint32_t lc = l * 3u + c;
            val[l] = grain_draw(dl[l] + q.dmin_l[lc], q.sat_d[lc], q.count[lc], q.uniformity[c], pixel,
                                SPK_STREAM_GRAIN(c, l), q.seed,
                                q.counts_out ? q.counts_out + size_t(pixel) * 9 + c * 3 + l : nullptr);
        }
        float G = ((0.0f + val[0]) + val[1]) + val[2];
        if (q.shift) G = G * 1.0f + (-q.dmin_c[c]);
        out[o + c] = G;
    }
}

// ---------------------------------------------------------------------------------------------------
// develop with sub-layer grain (SUM mode), the draws compacted per warp.
//
// A pixel's nine Poisson draws take data-dependent paths: most PTRS draws end at the first attempt's
// squeeze, the rest need the logarithm test, further attempts or (lam < 10) the product method. Run
// per lane, a warp would wait on its slowest lane at every draw. Here each lane makes every draw's
// first attempt in lockstep; a draw the squeeze does not settle goes to a ring of deferred draws in the
// warp's shared memory, and whenever 32 are queued the whole warp finishes them, one per lane. Every
// draw consumes the same uniforms in the same order and with the same arithmetic as spk_poisson, so the
// counts are those of the per-lane sampler.

#ifndef SPKB_DEVELOP_WARPS
#define SPKB_DEVELOP_WARPS 4
#endif
constexpr uint32_t kDrawWarps = SPKB_DEVELOP_WARPS;  // warps per block
// resident blocks per SM the register allocation is held to (1: no cap)
#ifndef SPKB_DEVELOP_MIN_BLOCKS
#define SPKB_DEVELOP_MIN_BLOCKS 1
#endif
constexpr uint32_t kDrawRing = 64;  // holds the < 32 left over plus one draw's 32

struct DeferredDraw {
    float lam, b, a, vr;        // the squeeze's PTRS constants (kinds 1, 2); lam alone for kind 0
    float loglam, loginvalpha;  // the full test's constants, once formed (kTagInited)
    float V, k, us;             // the last attempt's full test, pending (kind 1)
    uint32_t w2, w3;            // words z, w of the last Philox block: the next attempt's uniforms when it is odd
    uint32_t tag;               // kind | kTagInited | stream << 3 | slot << 11 | next attempt << 20
};
// kinds: 0 product method (lam < 10 or NaN); 1 the last attempt needs the full test; 2 it was rejected.
// slot = draw * 32 + lane: the draw's pixel is the warp's first plus the lane.
constexpr uint32_t kResStride = kDrawWarps * 32;  // a draw's row in the block's lambda / result array
constexpr uint32_t kTagInited = 4u;
__device__ __forceinline__ uint32_t draw_tag(uint32_t kind, uint32_t stream, uint32_t slot, uint32_t next) {
    return kind | (stream << 3) | (slot << 11) | (next << 20);
}

// log(k!) for k = 0 .. kLgammaTable - 1, each the sampler's own spk_lgamma_k(k + 1) computed by this
// device once per process (k_lgamma_table): the full test's largest single cost, a table read instead.
constexpr uint32_t kLgammaTable = 4096;
__device__ float g_lgamma[kLgammaTable];

__global__ void k_lgamma_table() {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kLgammaTable) g_lgamma[k] = spk_lgamma_k(SPK_ADD(float(k), 1.0f));
}

// spk_ptrs_test with log(k!) from the table while k is in it (k >= 0 and integral here)
__device__ __forceinline__ int ptrs_test_table(const spk_ptrs* p, float V, float k, float us) {
    const float L = SPK_SUB(SPK_ADD(spk_logf(V), p->loginvalpha),
                            spk_logf(SPK_ADD(SPK_DIV(p->a, SPK_MUL(us, us)), p->b)));
    const float lg = k < float(kLgammaTable) ? g_lgamma[int(k)] : spk_lgamma_k(SPK_ADD(k, 1.0f));
    const float Rt = SPK_SUB(SPK_ADD(-p->lam, SPK_MUL(k, p->loglam)), lg);
    return L <= Rt;
}

// One step of a deferred draw, exactly as spk_ptrs_from runs it: the last attempt's pending full test
// (kind 1), then, unless that accepted, the next attempt's uniforms and squeeze. Returns true once the
// draw's count is in res; false with e holding the state to queue again (kind 1 or 2, the next attempt).
// A product-method draw (kind 0) ends in one step. The test's constants (log lam, log 1 / alpha) are
// formed the first time a draw reaches the test and travel with it. pixel0: the warp's first pixel; res:
// the warp's results, draw k of lane j at res[k * kResStride + j].
__device__ __forceinline__ bool finish_step(DeferredDraw& e, uint32_t seed, uint32_t pixel0, float* res_warp) {
    const uint32_t kind = e.tag & 3u, stream = (e.tag >> 3) & 0xFFu, slot = (e.tag >> 11) & 0x1FFu;
    const uint32_t it = e.tag >> 20;
    const uint32_t pixel = pixel0 + (slot & 31u);
    float* res = res_warp + (slot >> 5) * kResStride + (slot & 31u);
    if (kind == 0u) {
        spk_stream g;
        spk_stream_init(&g, pixel, stream, seed);
        *res = spk_poisson_product(e.lam, &g);
        return true;
    }
    spk_ptrs p;
    p.lam = e.lam;
    p.b = e.b;
    p.a = e.a;
    p.vr = e.vr;
    bool inited = (e.tag & kTagInited) != 0u;
    if (kind == 1u) {
        if (inited) {
            p.loglam = e.loglam;
            p.loginvalpha = e.loginvalpha;
        } else {
            spk_ptrs_init_test(&p);
            e.loglam = p.loglam;
            e.loginvalpha = p.loginvalpha;
            inited = true;
        }
        if (ptrs_test_table(&p, e.V, e.k, e.us)) {
            *res = e.k;
            return true;
        }
    }
    if (it == 64u) {
        *res = SPK_FLOOR(p.lam);
        return true;
    }
    // attempt it takes uniforms 2 it and 2 it + 1: words x, y of Philox block it / 2 (it even, keeping z, w
    // for attempt it + 1) or the kept z, w (it odd)
    uint32_t wu = e.w2, wv = e.w3;
    if ((it & 1u) == 0u) {
        spk_u4 c4;
        c4.x = pixel;
        c4.y = stream;
        c4.z = it >> 1;
        c4.w = 0u;
        const spk_u4 b = spk_philox(c4, seed, 0u);
        wu = b.x;
        wv = b.y;
        e.w2 = b.z;
        e.w3 = b.w;
    }
    const float V = spk_uniform(wv);
    float k, us;
    const int r = spk_ptrs_squeeze(&p, spk_uniform(wu), V, &k, &us);
    if (r == SPK_PTRS_ACCEPT) {
        *res = k;
        return true;
    }
    e.V = V;
    e.k = k;
    e.us = us;
    e.tag = draw_tag(r == SPK_PTRS_TEST ? 1u : 2u, stream, slot, it + 1u) | (inited ? kTagInited : 0u);
    return false;
}

__global__ void __launch_bounds__(kDrawWarps * 32, SPKB_DEVELOP_MIN_BLOCKS) k_develop_layers(const float* __restrict__ exposure,
                                                                    float* __restrict__ out, uint32_t w,
                                                                    uint32_t blocks_per_row,
                                                                    const __grid_constant__ DevelopArgs q) {
    __shared__ DeferredDraw ring[kDrawWarps][kDrawRing];
    __shared__ float lam[9][kDrawWarps * 32], scale[9][kDrawWarps * 32];  // [c * 3 + l][thread]
    const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5, tid = threadIdx.x;
    const uint32_t y = blockIdx.x / blocks_per_row;
    const uint32_t x = (blockIdx.x - y * blocks_per_row) * (kDrawWarps * 32) + threadIdx.x;
    const bool live = x < w;
    const uint32_t pixel = y * q.width + x;
    const size_t o = 3 * (size_t(y) * w + x);

    // lambda and the count's scale of the nine draws, [c][l], kept in shared memory
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float dl[3] = {0.0f, 0.0f, 0.0f};
        if (live) {
            float L = log10f(fmaxf(exposure[o + c], 0.0f) + 1e-10f);
            if (q.chi) L = __fsub_rn(L, q.chi[o + c]);  // DIR couplers: the corrected log exposure, the y0 curve
            const float D = curve_lookup(q.cx, q.cinv, q.cy + size_t(c) * q.K, q.K, q.cgrid, L);
            layer_densities(q, uint32_t(c), q.positive ? -D : D, dl);
        }
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const int lc = l * 3 + c;
            float sat = 1.0f;
            lam[c * 3 + l][tid] =
                live ? spk_sublayer_lambda(dl[l] + q.dmin_l[lc], q.sat_d[lc], q.count[lc], q.uniformity[c], &sat)
                     : 0.0f;
            if (q.lam_out && live) q.lam_out[size_t(pixel) * 9 + c * 3 + l] = lam[c * 3 + l][tid];
            scale[c * 3 + l][tid] = SPK_MUL(q.unit[lc], sat);  // unit: SPK_DIV(sat_d, count), formed once
        }
    }

    DeferredDraw* ringw = ring[wi];
    // a draw's count replaces its lambda once the lockstep has read it: lam[k][tid] holds draw k of thread
    // tid until its attempt 0, then its count
    float* resw = &lam[0][wi * 32u];
    uint32_t head = 0, tail = 0;
#pragma unroll 1
    for (uint32_t k = 0; k < 9u; ++k) {
        const uint32_t stream = SPK_STREAM_GRAIN(k / 3u, k % 3u);
        bool defer = false;
        float value = 0.0f;
        DeferredDraw d{};
        uint32_t kind = 0u;
        const float lm = lam[k][tid];
        d.lam = lm;
        if (live) {
            if (lm >= 10.0f) {
                spk_ptrs p;
                spk_ptrs_init(&p, lm);
                spk_u4 c4;
                c4.x = pixel;
                c4.y = stream;
                c4.z = 0u;
                c4.w = 0u;
                const spk_u4 b0 = spk_philox(c4, q.seed, 0u);
                float kk, us;
                const int r = spk_ptrs_squeeze(&p, spk_uniform(b0.x), spk_uniform(b0.y), &kk, &us);
                if (r == SPK_PTRS_ACCEPT) {
                    value = kk;
                } else {
                    defer = true;
                    kind = r == SPK_PTRS_TEST ? 1u : 2u;
                    d.b = p.b;
                    d.a = p.a;
                    d.vr = p.vr;
                    d.V = spk_uniform(b0.y);
                    d.k = kk;
                    d.us = us;
                    d.w2 = b0.z;
                    d.w3 = b0.w;
                }
            } else {
                defer = true;
            }
        }
        const uint32_t mask = __ballot_sync(0xFFFFFFFFu, defer);
        if (defer) {
            d.tag = draw_tag(kind, stream, k * 32u + lane, 1u);
            ringw[(tail + __popc(mask & ((1u << lane) - 1u))) & (kDrawRing - 1u)] = d;
        } else {
            resw[k * kResStride + lane] = value;
        }
        tail += __popc(mask);
        // one step for 32 deferred draws at a time, the unfinished queued again behind the rest; after the
        // last draw, until none is left. The ring holds at most 63: fewer than 32 left over plus 32 queued.
        while (tail - head >= 32u || (k == 8u && tail != head)) {
            __syncwarp();
            const uint32_t n = min(tail - head, 32u);
            DeferredDraw e;
            bool again = false;
            if (lane < n) {
                e = ringw[(head + lane) & (kDrawRing - 1u)];
                again = !finish_step(e, q.seed, pixel - lane, resw);
            }
            head += n;
            __syncwarp();
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, again);
            if (again) ringw[(tail + __popc(m & ((1u << lane) - 1u))) & (kDrawRing - 1u)] = e;
            tail += __popc(m);
            __syncwarp();
        }
    }
    if (!live) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float val[3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const float cnt = resw[(c * 3 + l) * kResStride + lane];
            if (q.counts_out) q.counts_out[size_t(pixel) * 9 + c * 3 + l] = cnt;
            val[l] = SPK_MUL(cnt, scale[c * 3 + l][tid]);
        }
        float G = ((0.0f + val[0]) + val[1]) + val[2];
        if (q.shift) G = G * 1.0f + (-q.dmin_c[c]);
        out[o + c] = G;
    }
}

// ---------------------------------------------------------------------------------------------------
// encode: reference kernels/print.metal:129-156 and :350-366 (helpers in encode.cuh).

__global__ void k_encode(const float* __restrict__ rgb, const float* __restrict__ gpl, uint16_t* __restrict__ out,
                         uint32_t w, uint32_t h, const __grid_constant__ EncodeArgs e) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t i = 3 * (size_t(y) * w + x);
    float v0 = rgb[i], v1 = rgb[i + 1], v2 = rgb[i + 2];
    if (e.unsharp) {
        v0 = e.lincomb_a * v0 + e.lincomb_b * gpl[i];
        v1 = e.lincomb_a * v1 + e.lincomb_b * gpl[i + 1];
        v2 = e.lincomb_a * v2 + e.lincomb_b * gpl[i + 2];
    }
    edr_tone(e, v0, v1, v2);
    if (e.cctf_active) {
        float m0, m1, m2;
        mat_apply(e.m_nid, v0, v1, v2, m0, m1, m2);
        v0 = cctf_encode(m0, e.cctf_mode);
        v1 = cctf_encode(m1, e.cctf_mode);
        v2 = cctf_encode(m2, e.cctf_mode);
    }
    ushort4 p;
    p.x = encode16(v0);
    p.y = encode16(v1);
    p.z = encode16(v2);
    p.w = 65535;
    reinterpret_cast<ushort4*>(out)[size_t(y) * e.stride + x] = p;
}

// ---------------------------------------------------------------------------------------------------
// source copy: channels 3 or 4 -> interleaved RGB, non-finite -> 0 (reference src/session/session.cpp:164-168)

__global__ void k_source(const float* __restrict__ raw, float* __restrict__ out, size_t n, uint32_t channels) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float v = raw[i * channels + c];
        out[3 * i + c] = isfinite(v) ? v : 0.0f;
    }
}

// L2 flush: write a buffer larger than the L2 cache
__global__ void k_fill(uint4* p, size_t n, uint32_t v) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        p[i] = make_uint4(v, v, v, v);
}

// ---------------------------------------------------------------------------------------------------
// test kernels

__global__ void k_sampler_poisson(const float* lam, float* out, uint32_t n, uint32_t stream, uint32_t seed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = spk_poisson(lam[i], i, stream, seed);
}

// The print glare's field (reference kernels/fx_grain.metal:99-116 with same_all): one lognormal value
// per pixel, on stream 200 with the print seed, written to the three channels.
__global__ void k_glare_field(float* out, uint32_t n, float mean, float sd, uint32_t seed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = spk_lognormal(mean, sd, i, 200u, seed);
    out[3 * size_t(i)] = v;
    out[3 * size_t(i) + 1] = v;
    out[3 * size_t(i) + 2] = v;
}

__global__ void k_sampler_lognormal(float* out, uint32_t n, float mean, float sd, uint32_t stream, uint32_t seed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = spk_lognormal(mean, sd, i, stream, seed);
}

__global__ void k_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    spk_u4 c;
    c.x = ctr[4 * i];
    c.y = ctr[4 * i + 1];
    c.z = ctr[4 * i + 2];
    c.w = ctr[4 * i + 3];
    const spk_u4 r = spk_philox(c, key[2 * i], key[2 * i + 1]);
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
}

}  // namespace

// ---- launchers ------------------------------------------------------------------------------------

namespace {
thread_local LaunchHook* t_hook = nullptr;
std::atomic<uint64_t> g_launches{0};
}  // namespace

Probe::Probe(const char* name, cudaStream_t st) : s(st) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (t_hook) t_hook->before(name, s);
}
Probe::~Probe() {
    if (t_hook) t_hook->after(s);
}

unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0{}, q1{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000, cudaEnableDefault, &q0) != cudaSuccess ||
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault, &q1) != cudaSuccess ||
            !f0 || !f1)
            return;
        get_current = reinterpret_cast<GetCurrent>(f0);
        get_id = reinterpret_cast<GetId>(f1);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

void ensure_smem(const void* kernel, int bytes) {
    static std::mutex m;
    static std::map<std::pair<const void*, unsigned long long>, int> done;
    unsigned long long ctx = current_context_id();
    if (ctx == 0) {  // no context yet: make the device's primary one current first
        cudaFree(nullptr);
        ctx = current_context_id();
    }
    std::lock_guard<std::mutex> g(m);
    int& cur = done[{kernel, ctx}];
    if (ctx != 0 && bytes <= cur) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cur = bytes;
}

void set_launch_hook(LaunchHook* hook) { t_hook = hook; }
uint64_t launch_count() { return g_launches.load(); }

void expose(const float* rgb, float* h, const float* table4, const float* patches, const ExposeArgs& a,
            cudaStream_t s) {
    if (a.n == 0) return;
    Probe p("expose", s);
    const bool aligned = ((reinterpret_cast<uintptr_t>(rgb) | reinterpret_cast<uintptr_t>(h)) & 15u) == 0;
    if (patches && aligned) {
        k_expose_patch<<<div_up(div_up(a.n, 4), kExposeThreads), kExposeThreads, 0, s>>>(rgb, h, patches, a);
        return;
    }
    k_expose<<<div_up(a.n, 256), 256, 0, s>>>(rgb, h, reinterpret_cast<const float4*>(table4), a);
}

void iir_tangent(const float* in, const float* in_dot, float* work, float* work_dot, float* out, float* out_dot,
                 uint32_t w, uint32_t h, bool vertical, const IirCoefs& c, const IirCoefs& dc, cudaStream_t s) {
    const uint32_t lines = vertical ? 3u * w : 3u * h;
    if (lines == 0) return;
    Probe p("iir_tangent", s);
    // lines staged in shared memory where they fit, kTanSegs threads per line (strips of up to 10 rows or 4
    // pixel columns, at most 32 lines for the 256-thread CTA); the lines in global memory otherwise
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t n = vertical ? h : w;
    TangentMaps maps{};
    maps.L = uint32_t((n + kTanSegs - 1) / kTanSegs);
    for (int ch = 0; ch < 3; ++ch) {
        // the homogeneous one-step map A of (w1, w2, w3, t1, t2, t3), raised to the L-th power by squaring
        double A[36] = {0}, R[36] = {0}, T[36];
        A[0] = c.B1[ch], A[1] = c.B2[ch], A[2] = c.B3[ch];
        A[6] = 1.0;
        A[13] = 1.0;
        A[18] = dc.B1[ch], A[19] = dc.B2[ch], A[20] = dc.B3[ch], A[21] = c.B1[ch], A[22] = c.B2[ch], A[23] = c.B3[ch];
        A[27] = 1.0;
        A[34] = 1.0;
        for (int i = 0; i < 6; ++i) R[i * 7] = 1.0;
        auto mul = [&](const double* X, const double* Y, double* Z) {
            for (int r = 0; r < 6; ++r)
                for (int q2 = 0; q2 < 6; ++q2) {
                    double acc = 0.0;
                    for (int m = 0; m < 6; ++m) acc += X[r * 6 + m] * Y[m * 6 + q2];
                    T[r * 6 + q2] = acc;
                }
            for (int i = 0; i < 36; ++i) Z[i] = T[i];
        };
        for (uint32_t e = maps.L; e > 0; e >>= 1) {
            if (e & 1u) mul(R, A, R);
            mul(A, A, A);
        }
        for (int i = 0; i < 36; ++i) maps.AL[ch][i] = R[i];
    }
    for (uint32_t px : {10u, 8u, 4u, 2u, 1u}) {
        if (vertical && px > 4u) continue;
        const size_t smem = size_t(3 * px) * kTanSegs * 6 * sizeof(double) + 2 * n * (3 * px) * sizeof(float);
        if (smem > size_t(optin)) continue;
        ensure_smem(reinterpret_cast<const void*>(k_iir_tangent_seg), int(smem));
        const uint32_t ctas = div_up(vertical ? w : h, px);
        k_iir_tangent_seg<<<ctas, 256, smem, s>>>(in, in_dot, out, out_dot, w, h, vertical ? 1 : 0, px, c, dc, maps);
        return;
    }
    // a thread per line and few lines (3 per row or column): 32-thread CTAs spread them over more SMs
    k_iir_tangent<<<div_up(lines, 32), 32, 0, s>>>(in, in_dot, work, work_dot, out, out_dot, w, h, vertical ? 1 : 0, c,
                                                   dc);
}

void fir_v(const float* in, float* out, uint32_t w, uint32_t h, const FirTaps& t, cudaStream_t s) {
    const dim3 b(32, 8), g(div_up(w, 32), div_up(h, 8));
    Probe p("fir_v", s);
    k_fir_v<<<g, b, 0, s>>>(in, out, w, h, t);
}

void fir_h(const float* in, float* out, const float* acc, uint32_t w, uint32_t h, const FirTaps& t, int mode,
           const float weight[3], cudaStream_t s) {
    const dim3 b(32, 8), g(div_up(w, 32), div_up(h, 8));
    Probe p("fir_h", s);
    k_fir_h<<<g, b, 0, s>>>(in, out, acc, w, h, t, mode, weight[0], weight[1], weight[2]);
}

void iir_h(const float* in, float* out, uint32_t w, uint32_t h, const IirCoefs& c, cudaStream_t s) {
    Probe p("iir_h", s);
    k_iir_h<<<div_up(3 * h, 64), 64, 0, s>>>(in, out, w, h, c);
}

void iir_v(float* work, float* out, const float* acc, uint32_t w, uint32_t h, const IirCoefs& c, int mode,
           const float weight[3], cudaStream_t s) {
    Probe p("iir_v", s);
    k_iir_v<<<div_up(3 * w, 64), 64, 0, s>>>(work, out, acc, w, h, c, mode, weight[0], weight[1], weight[2]);
}

void lincomb(const float* x, const float* y, float* out, size_t pixels, const float a[3], const float b[3],
             cudaStream_t s) {
    if (pixels == 0) return;
    Probe p("lincomb", s);
    k_lincomb<<<unsigned((pixels + 255) / 256), 256, 0, s>>>(x, y, out, pixels, a[0], a[1], a[2], b[0], b[1], b[2]);
}

void copy(const float* x, float* out, size_t pixels, cudaStream_t s) {
    const size_t n = 3 * pixels;
    if (n == 0) return;
    Probe p("copy", s);
    k_copy<<<unsigned((n + 255) / 256), 256, 0, s>>>(x, out, n);
}

void develop_prepare(cudaStream_t s) {
    static std::mutex m;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> g(m);
    if (done[dev]) return;
    k_lgamma_table<<<div_up(kLgammaTable, 256), 256, 0, s>>>();
    // once written and waited for, every later launch on any stream reads the table
    if (cudaStreamSynchronize(s) == cudaSuccess && cudaGetLastError() == cudaSuccess) done[dev] = true;
}

void develop(const float* exposure, float* out, const DevelopArgs& a, uint32_t w, uint32_t h, cudaStream_t s) {
    if (uint64_t(w) * h == 0) return;
    if (a.grain && a.mode == 0) {
        develop_prepare(s);
        const uint32_t bx = div_up(w, kDrawWarps * 32);
        Probe p("develop_layers", s);
        k_develop_layers<<<bx * h, kDrawWarps * 32, 0, s>>>(exposure, out, w, bx, a);
        return;
    }
    const dim3 b(32, 4), g(div_up(w, 32), div_up(h, 4));
    Probe p("develop", s);
    k_develop<<<g, b, 0, s>>>(exposure, out, w, h, a);
}

void coupler_source(const float* exposure, float* chi, const CouplerArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    Probe p("coupler_source", s);
    k_coupler_source<<<div_up(a.n, 256), 256, 0, s>>>(exposure, chi, a);
}

void encode(const float* rgb, const float* g, uint16_t* out, uint32_t w, uint32_t h, const EncodeArgs& e,
            cudaStream_t s) {
    const dim3 b(32, 8), gr(div_up(w, 32), div_up(h, 8));
    Probe p("encode", s);
    k_encode<<<gr, b, 0, s>>>(rgb, g, out, w, h, e);
}

void source_copy(const float* raw, float* out, size_t pixels, uint32_t channels, cudaStream_t s) {
    if (pixels == 0) return;
    Probe p("source_copy", s);
    k_source<<<unsigned((pixels + 255) / 256), 256, 0, s>>>(raw, out, pixels, channels);
}

void fill(void* p, size_t bytes, uint32_t v, cudaStream_t s) {
    Probe pr("fill", s);
    k_fill<<<148 * 8, 256, 0, s>>>(static_cast<uint4*>(p), bytes / 16, v);
}

void sampler_poisson(const float* lam, float* out, uint32_t n, uint32_t stream, uint32_t seed, cudaStream_t s) {
    if (n == 0) return;
    Probe p("sampler_poisson", s);
    k_sampler_poisson<<<div_up(n, 128), 128, 0, s>>>(lam, out, n, stream, seed);
}

void glare_field(float* out, uint32_t pixels, float mean, float sd, uint32_t seed, cudaStream_t s) {
    Probe p("glare_field", s);
    k_glare_field<<<div_up(pixels, 256), 256, 0, s>>>(out, pixels, mean, sd, seed);
}

void sampler_lognormal(float* out, uint32_t n, float mean, float stddev, uint32_t stream, uint32_t seed,
                       cudaStream_t s) {
    if (n == 0) return;
    Probe p("sampler_lognormal", s);
    k_sampler_lognormal<<<div_up(n, 128), 128, 0, s>>>(out, n, mean, stddev, stream, seed);
}

void philox_blocks(const uint32_t* ctr, const uint32_t* key, uint32_t* out, uint32_t n, cudaStream_t s) {
    if (n == 0) return;
    Probe p("philox", s);
    k_philox<<<div_up(n, 128), 128, 0, s>>>(ctr, key, out, n);
}

}  // namespace spkb::dev
