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
#include "launch.hpp"
#include "print_common.cuh"

namespace spkb::dev {

namespace {

constexpr uint32_t kPrintThreads = 128;

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
        float x = fmaxf(k ? X.y : X.x, 0.0f) + kTiny;
        float y = fmaxf(k ? Y.y : Y.x, 0.0f) + kTiny;
        float z = fmaxf(k ? Z.y : Z.x, 0.0f) + kTiny;
        apply_levels(a, x, y, z);
        add_glare(a, size_t(p0 + k), x, y, z);
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
