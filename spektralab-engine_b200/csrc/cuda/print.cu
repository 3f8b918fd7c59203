// print: negative density -> linear output RGB. Reference kernels/print.metal:29-127 (CAM16 helpers)
// and :165-317 (enlarger integral, gain, paper curve, scan integral, output matrix, gamut compression).
//
// Two pixels per thread. The two spectral integrals (81 wavelengths each) run on packed f32x2
// arithmetic, the pair of pixels in the two halves: per wavelength three packed FMA form the exponent
// e = -log2(10) sum_c d_c eps_c, two ex2 give T = 2^e, and three packed FMA accumulate T w_k. The tables
// come from the kernel's constant bank with each value duplicated into both halves, and the base
// density is folded into the weights on the host (w_k = wt_k 10^-beta), so T = 10^-(d.eps + beta)
// enters the sum with the reference's meaning. The per-pixel remainder (gain, paper curve, gamut) is
// scalar, one pixel after the other.
//
// Precision: every spectral value, exponent and transmittance is binary32 with ex2.approx (relative
// error about 2^-22); the gamut stage takes the PTX approximate divide and square root and the
// special-function power (encode.cuh). The render tests hold the 16-bit output to +-1 LSB of the binary64
// oracle and of the reference's precise build.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../kernel_args.h"
#include "encode.cuh"
#include "launch.hpp"
#include "lookup.cuh"

namespace spkb::dev {

namespace {

constexpr float kLog10Of2 = 0.30102999566398120f;
constexpr float kLog2Of10 = 3.321928094887362f;
constexpr float kTiny = 1e-10f;
constexpr uint32_t kPrintThreads = 128;

__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
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
__device__ __forceinline__ float2 dup(const F32Pair& p) { return make_float2(p.x, p.y); }

// R_k for a pair of pixels: sum over l of 2^(e(l)) w_k(l), ascending l
__device__ __forceinline__ void spectral2(const SpectralPairs& t, float2 d0, float2 d1, float2 d2, float2& r0,
                                          float2& r1, float2& r2) {
    r0 = r1 = r2 = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int l = 0; l < SPKB_NL; ++l) {
        const float2 e =
            __ffma2_rn(d2, dup(t.e[3 * l + 2]), __ffma2_rn(d1, dup(t.e[3 * l + 1]), __fmul2_rn(d0, dup(t.e[3 * l]))));
        const float2 T = make_float2(ex2_ftz(e.x), ex2_ftz(e.y));
        r0 = __ffma2_rn(T, dup(t.w[3 * l]), r0);
        r1 = __ffma2_rn(T, dup(t.w[3 * l + 1]), r1);
        r2 = __ffma2_rn(T, dup(t.w[3 * l + 2]), r2);
    }
}

// log10(max(x, 0) + 1e-10) as log2 on the special-function unit times log10 2 (absolute error about
// 2^-22 on the log-exposure axis)
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
    const float et = 0.25f * (cosf(h + 2.0f) + 3.8f);
    const float A = (((2.0f * ra + ga) + ba * RCP(20.0f)) - 0.305f) * q.n_bb;
    const float ratio = A * q.inv_a_w;
    const float J = (100.0f * sgnf(ratio)) * powm(fabsf(ratio), cz);
    const float den = (ra + ga) + (21.0f * ba) * RCP(20.0f);
    const float t = den != 0.0f ? fdiv(((((50000.0f / 13.0f) * q.n_c) * q.n_cb) * et) * fsqrt(a * a + bb * bb), den)
                                : 0.0f;
    const float C = t > 0.0f ? (powm(t, 0.9f) * fsqrt(fabsf(J) * RCP(100.0f))) * chroma_k : 0.0f;
    const float M = C * f_l_qrt;
    const float Mp = logf(1.0f + 0.0228f * M) * RCP(0.0228f);
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
    const float Mi = (expf(0.0228f * Mn) - 1.0f) * RCP(0.0228f);
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
        float sh, ch;
        sincosf(h, &sh, &ch);
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

// pixels p0 and p0 + 1 (when p0 + 1 < n) of one frame
__device__ __forceinline__ void print_pair(const PrintArgs& a, const float* __restrict__ neg, float* __restrict__ rgb,
                                           uint32_t p0, uint32_t n) {
    const bool two = p0 + 1 < n;
    const float* s0 = neg + 3 * size_t(p0);
    const float* s1 = two ? s0 + 3 : s0;
    float2 d0 = make_float2(s0[0], s1[0]), d1 = make_float2(s0[1], s1[1]), d2 = make_float2(s0[2], s1[2]);
    if (a.printed) {
        float2 r0, r1, r2;
        spectral2(a.enl, d0, d1, d2, r0, r1, r2);
        d0 = make_float2(print_density(a, 0, r0.x), print_density(a, 0, r0.y));
        d1 = make_float2(print_density(a, 1, r1.x), print_density(a, 1, r1.y));
        d2 = make_float2(print_density(a, 2, r2.x), print_density(a, 2, r2.y));
    }
    float2 X, Y, Z;
    spectral2(a.scan, d0, d1, d2, X, Y, Z);
#pragma unroll 1
    for (uint32_t k = 0; k < 2u; ++k) {
        if (k == 1u && !two) break;
        const float x = fmaxf(k ? X.y : X.x, 0.0f) + kTiny;
        const float y = fmaxf(k ? Y.y : Y.x, 0.0f) + kTiny;
        const float z = fmaxf(k ? Z.y : Z.x, 0.0f) + kTiny;
        float r, g, b;
        mat_apply(a.to_rgb, x, y, z, r, g, b);
        gamut(a, r, g, b);
        float* o = rgb + 3 * size_t(p0 + k);
        o[0] = r;
        o[1] = g;
        o[2] = b;
    }
}

__global__ void __launch_bounds__(kPrintThreads) k_print(const float* __restrict__ neg, float* __restrict__ rgb,
                                                         const __grid_constant__ PrintArgs a) {
    const uint32_t p0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (p0 >= a.n) return;
    print_pair(a, neg, rgb, p0, a.n);
}

// The print stage of many frames in one persistent launch. Work item i covers `item_px` pixels of frame
// item_frame[i] from pixel item_first[i]; the CTAs take items i = blockIdx.x, blockIdx.x + gridDim.x, ...
// (items are ordered by frame, so a CTA mostly stays on one frame) and stage the frame's arguments in
// shared memory when the frame changes.
__global__ void __launch_bounds__(kPrintThreads) k_print_batch(const BatchPrintFrame* __restrict__ frames,
                                                               const uint32_t* __restrict__ item_frame,
                                                               const uint32_t* __restrict__ item_first,
                                                               uint32_t n_items, uint32_t item_px) {
    __shared__ __align__(16) PrintArgs sa;
    __shared__ const float* s_neg;
    __shared__ float* s_rgb;
    uint32_t cur = 0xFFFFFFFFu;
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
        const uint32_t f = item_frame[it];
        if (f != cur) {
            __syncthreads();
            const uint4* src = reinterpret_cast<const uint4*>(&frames[f].args);
            uint4* dst = reinterpret_cast<uint4*>(&sa);
            for (uint32_t i = threadIdx.x; i < sizeof(PrintArgs) / 16; i += blockDim.x) dst[i] = src[i];
            if (threadIdx.x == 0) {
                s_neg = frames[f].neg;
                s_rgb = frames[f].rgb;
            }
            __syncthreads();
            cur = f;
        }
        const uint32_t first = item_first[it];
        for (uint32_t p0 = first + 2 * threadIdx.x; p0 < min(first + item_px, sa.n); p0 += 2 * blockDim.x)
            print_pair(sa, s_neg, s_rgb, p0, sa.n);
    }
}

}  // namespace

void print(const float* neg, float* rgb, const PrintArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    const uint32_t threads = (a.n + 1) / 2;
    Probe p("print", s);
    k_print<<<(threads + kPrintThreads - 1) / kPrintThreads, kPrintThreads, 0, s>>>(neg, rgb, a);
}

void print_batch(const BatchPrintFrame* frames, const uint32_t* item_frame, const uint32_t* item_first,
                 uint32_t n_items, uint32_t item_px, uint32_t ctas, cudaStream_t s) {
    if (n_items == 0) return;
    Probe p("print_batch", s);
    k_print_batch<<<ctas, kPrintThreads, 0, s>>>(frames, item_frame, item_first, n_items, item_px);
}

}  // namespace spkb::dev
