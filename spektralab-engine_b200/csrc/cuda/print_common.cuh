// The per-pixel stages of the print around its two spectral integrals, shared by the print kernels
// (print.cu: binary32 on the CUDA cores; print_tc.cu: the spectral-mode kernel): gain and paper curve
// (reference kernels/print.metal:192-232) and the CAM16-UCS gamut compression (print.metal:51-127,
// :267-317), with the approximate special-function arithmetic described in print.cu.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../kernel_args.h"
#include "encode.cuh"
#include "lookup.cuh"

namespace spkb::dev {
namespace {

constexpr float kLog10Of2 = 0.30102999566398120f;
constexpr float kLog2Of10 = 3.321928094887362f;
constexpr float kTiny = 1e-10f;

__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// 2^x for a pair of binary32 values on the FMA pipe: a stand-in for ex2.approx on part of the print's
// wavelengths, where the special-function unit is the busiest pipe. Method: Cody and Waite's argument
// reduction x = j + r with j = rint(x) from the 1.5 * 2^23 addition and r = x - j in [-1/2, 1/2] (both
// exact); 2^r by the degree-6 polynomial of least maximum relative error on [-1/2, 1/2] (Remez exchange,
// coefficients rounded to binary32; with the binary32 Horner steps the relative error stays below 8e-8,
// under ex2.approx's); 2^j added to the result's exponent field. x is clamped to [-126, 126] first, so the
// result is a normal number (the print's exponents lie in [-60, 0]).
__device__ __forceinline__ float2 exp2_poly2(float2 x) {
    constexpr float kShift = 12582912.0f;  // 1.5 * 2^23: x + kShift rounds x to an integer in its low bits
    x.x = fminf(fmaxf(x.x, -126.0f), 126.0f);
    x.y = fminf(fmaxf(x.y, -126.0f), 126.0f);
    const float2 t = __fadd2_rn(x, make_float2(kShift, kShift));
    const float2 j = __fadd2_rn(t, make_float2(-kShift, -kShift));
    const float2 r = __ffma2_rn(j, make_float2(-1.0f, -1.0f), x);
    float2 p = make_float2(0x1.41d334p-13f, 0x1.41d334p-13f);
    p = __ffma2_rn(p, r, make_float2(0x1.5f456ap-10f, 0x1.5f456ap-10f));
    p = __ffma2_rn(p, r, make_float2(0x1.3b2dbcp-7f, 0x1.3b2dbcp-7f));
    p = __ffma2_rn(p, r, make_float2(0x1.c6aed4p-5f, 0x1.c6aed4p-5f));
    p = __ffma2_rn(p, r, make_float2(0x1.ebfbdap-3f, 0x1.ebfbdap-3f));
    p = __ffma2_rn(p, r, make_float2(0x1.62e430p-1f, 0x1.62e430p-1f));
    p = __ffma2_rn(p, r, make_float2(1.0f, 1.0f));
    // the low bits of t hold j in two's complement; shifted to the exponent field they scale p by 2^j
    return make_float2(__int_as_float(__float_as_int(p.x) + (__float_as_int(t.x) << 23)),
                       __int_as_float(__float_as_int(p.y) + (__float_as_int(t.y) << 23)));
}

__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// a / b with PTX div.approx (2 ulp for |b| in [2^-126, 2^126]); a / 0 = +-inf, 0 / 0 = NaN
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float fsqrt(float x) {
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// log10(max(x, 0) + 1e-10) as log2 on the special-function unit times log10 2 (absolute error about
// 2^-22 on the log-exposure axis)
// Scanner levels (reference kernels/print.metal:234-246), each operation rounded on its own.
__device__ __forceinline__ void apply_levels(const PrintArgs& a, float& x, float& y, float& z) {
    if (!a.levels) return;
    const float Yp = fminf(fmaxf(__fadd_rn(__fmul_rn(a.levels_m, y), a.levels_q), 0.0f), 1.0f);
    const float s = __fdiv_rn(Yp, __fadd_rn(y, kTiny));
    x = __fmul_rn(s, x);
    y = __fmul_rn(s, y);
    z = __fmul_rn(s, z);
}

// Print glare (reference kernels/fx_glare.metal:12-22): xyz_c + (F / 100) tint_c for the field value F of
// pixel p, each operation rounded on its own.
__device__ __forceinline__ void add_glare(const PrintArgs& a, size_t p, float& x, float& y, float& z) {
    if (!a.glare) return;
    const float f = __fdiv_rn(a.glare[3 * p], 100.0f);
    x = __fadd_rn(x, __fmul_rn(f, a.glare_tint[0]));
    y = __fadd_rn(y, __fmul_rn(f, a.glare_tint[1]));
    z = __fadd_rn(z, __fmul_rn(f, a.glare_tint[2]));
}

__device__ __forceinline__ float log10_floor(float x) { return lg2_approx(fmaxf(x, 0.0f) + kTiny) * kLog10Of2; }

__device__ __forceinline__ float paper_lookup(const float* __restrict__ tab, uint32_t K, const AxisGrid& g,
                                              uint32_t c, float v) {
    if (isnan(v)) return v;
    const float* x = tab;
    const float* r = tab + K;
    const float* y = tab + 2 * K;
    if (v <= __ldg(x)) return __ldg(y + c);
    if (v >= __ldg(x + K - 1)) return __ldg(y + 3 * (K - 1) + c);
    const uint32_t j = axis_index(x, 1, K, g, v);
    const float y0 = __ldg(y + 3 * j + c);
    return y0 + ((v - __ldg(x + j)) * __ldg(r + j)) * (__ldg(y + 3 * (j + 1) + c) - y0);
}

// A division by a per-frame or literal constant is a product with its binary32 reciprocal (formed on the
// host, or folded by the compiler): as accurate as the approximate divide and no special-function op.
#define RCP(x) (1.0f / (x))

// 1: the gamut stage's cos, sin, log and exp on the special-function unit (__sincosf, __logf, __expf)
#ifndef SPKB_GAMUT_FAST
#define SPKB_GAMUT_FAST 0
#endif

__device__ __forceinline__ float knee(float d, float tau, float lim, float p, float inv_span, float inv_p) {
    if (d <= tau) return d;
    const float x = (d - tau) * inv_span;
    return tau + (lim - tau) * fdiv(x, powm(1.0f + powm(x, p), inv_p));
}

__device__ __forceinline__ float post_adapt(float v, float f_l) {
    const float f = powm((f_l * fabsf(v)) * RCP(100.0f), 0.42f);
    return fdiv((400.0f * sgnf(v)) * f, 27.13f + f) + 0.1f;
}

// CAM16-UCS gamut compression of one linear output RGB (print.metal:51-127, :267-317): forward to
// J', M', h; lightness knee; chroma knee against C_max(J', h); guarded inverse.
__device__ __forceinline__ void gamut(const PrintArgs& pa, float& r, float& g, float& b) {
    const Cam16Args& q = pa.cam;
    const float cz = q.cz, inv_cz = q.inv_cz, f_l_qrt = q.f_l_qrt, chroma_k = q.chroma_k;
    const float hundred_over_f_l = q.hundred_over_f_l;
    float X, Y, Z;
    mat_apply(q.m_to_xyz, r, g, b, X, Y, Z);
    float R16, G16, B16;
    mat_apply(q.m16, 100.0f * X, 100.0f * Y, 100.0f * Z, R16, G16, B16);
    const float ra = post_adapt(q.d_rgb[0] * R16, q.f_l);
    const float ga = post_adapt(q.d_rgb[1] * G16, q.f_l);
    const float ba = post_adapt(q.d_rgb[2] * B16, q.f_l);
    const float a = (ra - (12.0f * ga) * RCP(11.0f)) + ba * RCP(11.0f);
    const float bb = ((ra + ga) - 2.0f * ba) * RCP(9.0f);
    const float h = atan2f(bb, a);
#if SPKB_GAMUT_FAST
    // cos(h + 2) from the special-function sine and cosine of h in [-pi, pi]
    float sh_h, ch_h;
    __sincosf(h, &sh_h, &ch_h);
    const float et = 0.25f * ((ch_h * -0.41614683654714241f - sh_h * 0.90929742682568170f) + 3.8f);
#else
    const float et = 0.25f * (cosf(h + 2.0f) + 3.8f);
#endif
    const float A = (((2.0f * ra + ga) + ba * RCP(20.0f)) - 0.305f) * q.n_bb;
    const float ratio = A * q.inv_a_w;
    const float J = (100.0f * sgnf(ratio)) * powm(fabsf(ratio), cz);
    const float den = (ra + ga) + (21.0f * ba) * RCP(20.0f);
    const float t = den != 0.0f ? fdiv(((((50000.0f / 13.0f) * q.n_c) * q.n_cb) * et) * fsqrt(a * a + bb * bb), den)
                                : 0.0f;
    const float C = t > 0.0f ? (powm(t, 0.9f) * fsqrt(fabsf(J) * RCP(100.0f))) * chroma_k : 0.0f;
    const float M = C * f_l_qrt;
#if SPKB_GAMUT_FAST
    const float Mp = __logf(1.0f + 0.0228f * M) * RCP(0.0228f);
#else
    const float Mp = logf(1.0f + 0.0228f * M) * RCP(0.0228f);
#endif
    float Jp = fdiv(1.7f * J, 1.0f + 0.007f * J);
    if (q.lc_active != 0u) {
        float Ln = Jp * q.inv_j_white;
        if (Ln > q.lc[0]) {
            Ln = knee(Ln, q.lc[0], q.lc[1], q.lc[2], q.lc_inv_span, q.lc_inv_p);
            Jp = Ln * q.j_white;
        }
    }
    // C_max(J', h), bilinear with hue wrap
    const float Jc = fminf(fmaxf(Jp, q.j_first), q.j_last);
    const float u = ((Jc - q.j_first) * q.inv_j_span) * float(q.rows - 1);
    int l0 = int(floorf(u));
    l0 = l0 < 0 ? 0 : (l0 > int(q.rows) - 2 ? int(q.rows) - 2 : l0);
    const float fl = u - float(l0);
    const float v = (h - q.h_first) * q.inv_h_step;
    const float vf = floorf(v);
    const int cols = int(q.cols);
    int h0 = int(vf) % cols;
    if (h0 < 0) h0 += cols;
    const int h1 = h0 == cols - 1 ? 0 : h0 + 1;
    const float fh = v - vf;
    const float t00 = __ldg(pa.cmax + l0 * cols + h0), t01 = __ldg(pa.cmax + l0 * cols + h1);
    const float t10 = __ldg(pa.cmax + (l0 + 1) * cols + h0), t11 = __ldg(pa.cmax + (l0 + 1) * cols + h1);
    const float cm = (1.0f - fl) * ((1.0f - fh) * t00 + fh * t01) + fl * ((1.0f - fh) * t10 + fh * t11);
    const float cs = fmaxf(cm, 1e-9f);
    float dch = fdiv(Mp, cs);
    if (dch > 0.0f) dch = knee(dch, q.knee[0], q.knee[1], q.knee[2], q.knee_inv_span, q.knee_inv_p);
    const float Mn = dch * cs;
    // guarded inverse
#if SPKB_GAMUT_FAST
    const float Mi = (__expf(0.0228f * Mn) - 1.0f) * RCP(0.0228f);
#else
    const float Mi = (expf(0.0228f * Mn) - 1.0f) * RCP(0.0228f);
#endif
    const float Ji = fdiv(Jp, 1.7f - 0.007f * Jp);
    const float Ci = Mi * q.inv_f_l_qrt;
    const float Ai = (q.a_w * sgnf(Ji)) * powm(fabsf(Ji * RCP(100.0f)), inv_cz);
    const float sq = fsqrt(fabsf(Ji) * RCP(100.0f));
    const float ti = (sq > 0.0f && Ci > 0.0f) ? powm(fdiv(Ci, sq * chroma_k), 1.0f / 0.9f) : 0.0f;
    const float p2 = Ai * q.inv_n_bb + 0.305f;
    const float p3 = 21.0f / 20.0f;
    float ai = 0.0f, bi = 0.0f;
    if (ti != 0.0f) {
        const float p1 = fdiv((((50000.0f / 13.0f) * q.n_c) * q.n_cb) * et, ti);
#if SPKB_GAMUT_FAST
        const float sh = sh_h, ch = ch_h;
#else
        float sh, ch;
        sincosf(h, &sh, &ch);
#endif
        if (fabsf(sh) >= fabsf(ch)) {
            const float rs = fdiv(1.0f, sh);
            const float p4 = p1 * rs;
            bi = fdiv((p2 * (2.0f + p3)) * (460.0f / 1403.0f),
                      ((p4 + ((2.0f + p3) * (220.0f / 1403.0f)) * (ch * rs)) - 27.0f / 1403.0f) +
                          p3 * (6300.0f / 1403.0f));
            ai = (bi * ch) * rs;
        } else {
            const float rc = fdiv(1.0f, ch);
            const float p5 = p1 * rc;
            ai = fdiv((p2 * (2.0f + p3)) * (460.0f / 1403.0f),
                      (p5 + (2.0f + p3) * (220.0f / 1403.0f)) - (27.0f / 1403.0f - p3 * (6300.0f / 1403.0f)) * (sh * rc));
            bi = (ai * sh) * rc;
        }
    }
    const float xa[3] = {((460.0f * p2 + 451.0f * ai) + 288.0f * bi) * RCP(1403.0f),
                         ((460.0f * p2 - 891.0f * ai) - 261.0f * bi) * RCP(1403.0f),
                         ((460.0f * p2 - 220.0f * ai) - 6300.0f * bi) * RCP(1403.0f)};
    float rc3[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float vv = xa[i] - 0.1f;
        const float av = fabsf(vv);
        const float beta = av >= 400.0f ? 0.0f : fdiv(27.13f * av, 400.0f - av);
        rc3[i] = ((hundred_over_f_l * sgnf(vv)) * powm(beta, 1.0f / 0.42f)) * q.inv_d_rgb[i];
    }
    float x100, y100, z100;
    mat_apply(q.m16_inv, rc3[0], rc3[1], rc3[2], x100, y100, z100);
    mat_apply(q.m_to_rgb, x100 * RCP(100.0f), y100 * RCP(100.0f), z100 * RCP(100.0f), r, g, b);
}

// the print gain and paper curve of one pixel (print.metal:192-232): l := log10(max(R g + o, 0) + 1e-10),
// l := log10(max(10^l k, 0) + 1e-10), d := paper(l)
__device__ __forceinline__ float print_density(const PrintArgs& a, uint32_t c, float R) {
    float l = log10_floor(R * a.g[c] + a.o[c]);
    l = log10_floor(ex2_ftz(l * kLog2Of10) * a.k_gain);
    return paper_lookup(a.paper, a.paper_K, a.paper_grid, c, l);
}

}  // namespace
}  // namespace spkb::dev
