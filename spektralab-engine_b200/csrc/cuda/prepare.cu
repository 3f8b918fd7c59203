// The steps before the film path: the tier downscale of the frame, and the input transfer decode with
// the crop / rotation / quarter turn / flip geometry.
//
// Tier downscale (reference src/session/tiers.cpp:137-183 and kernels/session.metal:19-91): a vertical
// Gaussian prefilter, a horizontal one, then a bilinear sample from exact-integer index tables, all in
// binary32 with explicit fused multiply-adds in ascending tap order (so the bits do not depend on how a
// compiler contracts). Here the vertical pass runs over the frame and the horizontal pass is evaluated
// only at the four points each output pixel's bilinear sample reads, fused with the blend: the same
// values as the reference's full-resolution horizontal pass, without writing and re-reading it.
//
// Decode + geometry (reference kernels/film.metal:104-173): the transfer function per element, then the
// bilinear resample at a double-float source coordinate. Both run in one pass over the output; each of
// the four taps is decoded before the blend, which is the value the decode pass would have stored.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"
#include "launch.hpp"

namespace spkb::dev {

namespace {

inline unsigned div_up(size_t a, unsigned b) { return unsigned((a + b - 1) / b); }

// "c b | a b c d | c b": period 2 (n - 1); n == 1 -> 0 (reference src/util/numeric.cpp mirror_index)
__device__ __forceinline__ int mirror_index(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * (n - 1);
    int m = i % period;
    if (m < 0) m += period;
    return m < n ? m : period - m;
}

__global__ void k_tier_blur_v(const float* __restrict__ src, float* __restrict__ dst,
                              const __grid_constant__ TierBlurArgs a) {
    extern __shared__ float taps[];
    const int r = a.r;
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i <= 2 * r; i += blockDim.x * blockDim.y) taps[i] = a.taps[i];
    __syncthreads();
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f;
    for (int k = -r; k <= r; ++k) {
        const int yy = mirror_index(int(y) + k, int(a.h));
        const float wk = taps[k + r];
        const float* p = src + 3 * (size_t(yy) * a.w + x);
        acc0 = __fmaf_rn(wk, p[0], acc0);
        acc1 = __fmaf_rn(wk, p[1], acc1);
        acc2 = __fmaf_rn(wk, p[2], acc2);
    }
    float* q = dst + 3 * (size_t(y) * a.w + x);
    q[0] = acc0;
    q[1] = acc1;
    q[2] = acc2;
}

// the horizontal prefilter of plane v (in_w wide) at (x, y)
__device__ __forceinline__ void blur_h_at(const float* __restrict__ v, const float* taps, int rx, uint32_t in_w,
                                          uint32_t x, uint32_t y, float o[3]) {
    const float* row = v + 3 * size_t(y) * in_w;
    if (rx == 0) {
        o[0] = row[3 * x];
        o[1] = row[3 * x + 1];
        o[2] = row[3 * x + 2];
        return;
    }
    float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f;
    for (int k = -rx; k <= rx; ++k) {
        const int xx = mirror_index(int(x) + k, int(in_w));
        const float wk = taps[k + rx];
        const float* p = row + 3 * xx;
        acc0 = __fmaf_rn(wk, p[0], acc0);
        acc1 = __fmaf_rn(wk, p[1], acc1);
        acc2 = __fmaf_rn(wk, p[2], acc2);
    }
    o[0] = acc0;
    o[1] = acc1;
    o[2] = acc2;
}

__global__ void k_tier_resample(const float* __restrict__ v, float* __restrict__ dst,
                                const __grid_constant__ TierResampleArgs a) {
    extern __shared__ float taps[];
    const int rx = a.rx;
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i <= 2 * rx; i += blockDim.x * blockDim.y)
        taps[i] = a.taps_x[i];
    __syncthreads();
    const uint32_t ox = blockIdx.x * blockDim.x + threadIdx.x, oy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ox >= a.out_w || oy >= a.out_h) return;
    const uint32_t x0 = a.xi[2 * ox], x1 = a.xi[2 * ox + 1];
    const uint32_t y0 = a.yi[2 * oy], y1 = a.yi[2 * oy + 1];
    const float tx = a.xt[ox], ty = a.yt[oy];
    float pa[3], pb[3], pd[3], pe[3];
    blur_h_at(v, taps, rx, a.in_w, x0, y0, pa);
    blur_h_at(v, taps, rx, a.in_w, x1, y0, pb);
    blur_h_at(v, taps, rx, a.in_w, x0, y1, pd);
    blur_h_at(v, taps, rx, a.in_w, x1, y1, pe);
    float* q = dst + 3 * (size_t(oy) * a.out_w + ox);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float top = __fmaf_rn(tx, __fsub_rn(pb[c], pa[c]), pa[c]);
        const float bot = __fmaf_rn(tx, __fsub_rn(pe[c], pd[c]), pd[c]);
        q[c] = __fmaf_rn(ty, __fsub_rn(bot, top), top);
    }
}

// ---- decode + geometry -----------------------------------------------------------------------------

// The transfer functions' inverses (reference kernels/film.metal:104-142). The powers are evaluated in
// binary64 and rounded once, which gives the correctly rounded binary32 power in all but rare ties.
__device__ __forceinline__ float decode_one(float v, const PrepareArgs& q) {
    switch (q.mode) {
        case 0: {  // sRGB
            if (v <= 0.040449936f) return __fdiv_rn(v, 12.92f);
            const float u = __fdiv_rn(__fadd_rn(v, 0.055f), 1.055f);
            return copysignf(float(pow(double(fabsf(u)), double(2.4f))), u);
        }
        case 1:  // ProPhoto
            return v < 16.0f / 512.0f ? __fdiv_rn(v, 16.0f) : float(pow(double(v), double(1.8f)));
        case 2:  // Adobe
            return float(pow(double(v), double(563.0f / 256.0f)));
        case 3: {  // BT.709
            if (v < q.bt709_bp) return __fdiv_rn(v, 4.5f);
            const float u = __fdiv_rn(__fadd_rn(v, 0.099f), 1.099f);
            return copysignf(float(pow(double(fabsf(u)), double(q.bt709_exp))), u);
        }
        default:
            return v;
    }
}

struct F2 {
    float hi, lo;
};

// Knuth's two-sum and the double-float sum of the reference's geometry kernel, each operation rounded
// to nearest on its own.
__device__ __forceinline__ F2 two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return {s, e};
}
__device__ __forceinline__ F2 dd_add(F2 a, F2 b) {
    const F2 s = two_sum(a.hi, b.hi);
    const float e = __fadd_rn(s.lo, __fadd_rn(a.lo, b.lo));
    const float h = __fadd_rn(s.hi, e);
    const float l = __fsub_rn(e, __fsub_rn(h, s.hi));
    return {h, l};
}

// The clamped bilinear axis on the high part (reference kernels/film.metal:30-47).
__device__ __forceinline__ void geometry_axis(F2 f, uint32_t n, uint32_t& i0, uint32_t& i1, float& t) {
    const float hi = f.hi;
    if (hi <= 0.0f) {
        i0 = 0;
        t = 0.0f;
    } else if (hi >= float(n - 1)) {
        i0 = n - 1;
        t = 0.0f;
    } else {
        const float fl = floorf(hi);
        i0 = uint32_t(fl);
        t = __fadd_rn(__fsub_rn(hi, fl), f.lo);
        t = fminf(fmaxf(t, 0.0f), 1.0f);
    }
    i1 = min(i0 + 1, n - 1);
}

// P = sx u - hx, then (P cos, P sin); Q = sy v - hy, then (-(Q sin), Q cos): the plan's terms
__device__ __forceinline__ void put_u(const PrepareArgs& q, double u, double& tx, double& ty) {
    const double P = __dsub_rn(__dmul_rn(q.sx, u), q.hx);
    tx = __dmul_rn(P, q.ca);
    ty = __dmul_rn(P, q.sa);
}
__device__ __forceinline__ void put_v(const PrepareArgs& q, double v, double& tx, double& ty) {
    const double Q = __dsub_rn(__dmul_rn(q.sy, v), q.hy);
    tx = -__dmul_rn(Q, q.sa);
    ty = __dmul_rn(Q, q.ca);
}
__device__ __forceinline__ F2 split(double v) {
    const float hi = __double2float_rn(v);
    return {hi, __double2float_rn(__dsub_rn(v, double(hi)))};
}

__global__ void k_prepare(const float* __restrict__ src, float* __restrict__ dst, const __grid_constant__ PrepareArgs q) {
    const uint32_t ox = blockIdx.x * blockDim.x + threadIdx.x, oy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ox >= q.dst_w || oy >= q.dst_h) return;
    float* o = dst + 3 * (size_t(oy) * q.dst_w + ox);
    if (!q.geometry) {
        const float* p = src + 3 * (size_t(oy) * q.src_w + ox);
#pragma unroll
        for (int c = 0; c < 3; ++c) o[c] = q.decode ? decode_one(p[c], q) : p[c];
        return;
    }
    // the column's terms (u or v from the output column, by the quarter turn) and the row's
    double cxt, cyt, rxt, ryt;
    {
        double u0 = double(ox) + 0.5;
        if (q.flip_h) u0 = __dsub_rn(q.ow, u0);
        switch (q.quarter) {
            case 0: put_u(q, u0, cxt, cyt); break;
            case 1: put_v(q, __dsub_rn(q.ow, u0), cxt, cyt); break;
            case 2: put_u(q, __dsub_rn(q.ow, u0), cxt, cyt); break;
            default: put_v(q, u0, cxt, cyt); break;
        }
        double v0 = double(oy) + 0.5;
        if (q.flip_v) v0 = __dsub_rn(q.oh, v0);
        switch (q.quarter) {
            case 0: put_v(q, v0, rxt, ryt); break;
            case 1: put_u(q, v0, rxt, ryt); break;
            case 2: put_v(q, __dsub_rn(q.oh, v0), rxt, ryt); break;
            default: put_u(q, __dsub_rn(q.oh, v0), rxt, ryt); break;
        }
    }
    const F2 sx = dd_add(split(cxt), split(rxt));
    const F2 sy = dd_add(split(cyt), split(ryt));
    const F2 fx = dd_add(split(q.cx), sx);
    const F2 fy = dd_add(split(q.cy), sy);
    uint32_t x0, x1, y0, y1;
    float tx, ty;
    geometry_axis(fx, q.src_w, x0, x1, tx);
    geometry_axis(fy, q.src_h, y0, y1, ty);
    const float* pa = src + 3 * (size_t(y0) * q.src_w + x0);
    const float* pb = src + 3 * (size_t(y0) * q.src_w + x1);
    const float* pd = src + 3 * (size_t(y1) * q.src_w + x0);
    const float* pe = src + 3 * (size_t(y1) * q.src_w + x1);
    const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float va = pa[c], vb = pb[c], vd = pd[c], ve = pe[c];
        if (q.decode) {
            va = decode_one(va, q);
            vb = decode_one(vb, q);
            vd = decode_one(vd, q);
            ve = decode_one(ve, q);
        }
        const float top = __fadd_rn(__fmul_rn(va, ux), __fmul_rn(vb, tx));
        const float bot = __fadd_rn(__fmul_rn(vd, ux), __fmul_rn(ve, tx));
        o[c] = __fadd_rn(__fmul_rn(top, uy), __fmul_rn(bot, ty));
    }
}

}  // namespace

void tier_blur_v(const float* src, float* dst, const TierBlurArgs& a, cudaStream_t s) {
    const dim3 b(32, 8), g(div_up(a.w, 32), div_up(a.h, 8));
    const int smem = int((2 * a.r + 1) * sizeof(float));
    ensure_smem(reinterpret_cast<const void*>(k_tier_blur_v), smem);
    Probe p("tier_blur_v", s);
    k_tier_blur_v<<<g, b, smem, s>>>(src, dst, a);
}

void tier_resample(const float* v, float* dst, const TierResampleArgs& a, cudaStream_t s) {
    const dim3 b(32, 8), g(div_up(a.out_w, 32), div_up(a.out_h, 8));
    const int smem = int((2 * a.rx + 1) * sizeof(float));
    ensure_smem(reinterpret_cast<const void*>(k_tier_resample), smem);
    Probe p("tier_resample", s);
    k_tier_resample<<<g, b, smem, s>>>(v, dst, a);
}

void prepare(const float* src, float* dst, const PrepareArgs& a, cudaStream_t s) {
    const dim3 b(32, 8), g(div_up(a.dst_w, 32), div_up(a.dst_h, 8));
    Probe p("prepare", s);
    k_prepare<<<g, b, 0, s>>>(src, dst, a);
}

}  // namespace spkb::dev
