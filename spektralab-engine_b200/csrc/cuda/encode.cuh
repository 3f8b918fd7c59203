// Device helpers shared by the print and scanner kernels: a 3x3 matrix in the reference's bracketing,
// the output transfer functions and the 16-bit quantiser (reference kernels/print.metal:129-156,
// :350-366, print_shared.h).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace spkb::dev {
namespace {

__device__ __forceinline__ float sgnf(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

__device__ __forceinline__ void mat_apply(const float* m, float x, float y, float z, float& a, float& b, float& c) {
    a = (m[0] * x + m[1] * y) + m[2] * z;
    b = (m[3] * x + m[4] * y) + m[5] * z;
    c = (m[6] * x + m[7] * y) + m[8] * z;
}

// x^y for x >= 0 (NaN for x < 0, 0 for x = 0, y > 0) as 2^(y log2 x) on the special-function unit
// (PTX lg2.approx and ex2.approx, subnormals kept): relative error within about 2^-22 (1 + |y log2 x|),
// against 2 ulp for powf. Every use feeds a 16-bit output, whose 1 LSB is 2^-16 of full scale; the
// render tests hold the output to the binary64 oracle and to the reference's precise-math build.
__device__ __forceinline__ float powm(float x, float y) {
    float l, r;
    asm("lg2.approx.f32 %0, %1;" : "=f"(l) : "f"(x));
    asm("ex2.approx.f32 %0, %1;" : "=f"(r) : "f"(y * l));
    return r;
}

__device__ __forceinline__ float spowm(float v, float p) { return sgnf(v) * powm(fabsf(v), p); }

// mode 0 sRGB, 1 ProPhoto (ROMM), 2 Adobe RGB, 3 BT.709, otherwise identity
__device__ __forceinline__ float cctf_encode(float v, uint32_t mode) {
    switch (mode) {
        case 0: return v <= 0.0031308f ? 12.92f * v : 1.055f * spowm(v, 0.41666666666666669f) - 0.055f;
        case 1: return v < 0.001953125f ? 16.0f * v : powm(v, 0.55555555555555558f);
        case 2: return powm(v, 0.45470692717584371f);
        case 3: return v < 0.018f ? 4.5f * v : 1.099f * spowm(v, 0.45f) - 0.099f;
        default: return v;
    }
}

// floor(clamp(v, 0, 1) 65535 + 0.5); NaN -> 0
// The EDR tone map (reference kernels/print.metal:319-347): y = max(r_y . rgb, 0); outside [toe, shoulder]
// y' is 2 to the power of the target curve interpolated at the clamped log2 y; rgb times y' / (y + 1e-10).
// Each operation rounded on its own.
__device__ __forceinline__ void edr_tone(const EncodeArgs& e, float& r, float& g, float& b) {
    if (!e.edr) return;
    const float y = fmaxf(__fadd_rn(__fadd_rn(__fmul_rn(e.edr_r_y[0], r), __fmul_rn(e.edr_r_y[1], g)),
                                    __fmul_rn(e.edr_r_y[2], b)),
                          0.0f);
    float yp = y;
    if (y > 0.0f && (y < e.edr_toe || y > e.edr_shoulder)) {
        const uint32_t N = e.edr_n > 2u ? e.edr_n : 2u;
        const float u = __fmul_rn(fminf(fmaxf(__fdiv_rn(__fsub_rn(log2f(y), e.edr_lo), e.edr_span), 0.0f), 1.0f),
                                  float(N - 1));
        const uint32_t i0 = min(uint32_t(floorf(u)), N - 2);
        const float t = __fsub_rn(u, float(i0));
        yp = exp2f(__fadd_rn(__fmul_rn(__fsub_rn(1.0f, t), e.edr_tab[i0]), __fmul_rn(t, e.edr_tab[i0 + 1])));
    }
    const float den = __fadd_rn(y, 1e-10f);
    r = __fdiv_rn(__fmul_rn(r, yp), den);
    g = __fdiv_rn(__fmul_rn(g, yp), den);
    b = __fdiv_rn(__fmul_rn(b, yp), den);
}

__device__ __forceinline__ uint16_t encode16(float v) {
    if (isnan(v)) return 0;
    const float c = fminf(fmaxf(v, 0.0f), 1.0f);
    return uint16_t(floorf(c * 65535.0f + 0.5f));
}

}  // namespace
}  // namespace spkb::dev
