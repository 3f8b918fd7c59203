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

// 512 threads per CTA: the warps of a CTA start together and run the same fully unrolled spectral code
// close behind one another, so they share its instruction-cache lines (4K print 0.648 ms at 128 threads,
// 0.566 at 256, 0.527 at 512, outputs identical)
#ifndef SPKB_PRINT_THREADS
#define SPKB_PRINT_THREADS 512
#endif
constexpr uint32_t kPrintThreads = SPKB_PRINT_THREADS;

// Every kPolyEvery-th wavelength (l % kPolyEvery == kPolyEvery - 1) takes its 2^e from the FMA-pipe
// polynomial (exp2_poly2) instead of the special-function unit; 0: none. The split balances the two pipes.
#ifndef SPKB_PRINT_POLY_EVERY
#define SPKB_PRINT_POLY_EVERY 0
#endif
constexpr int kPolyEvery = SPKB_PRINT_POLY_EVERY;

// Packed pixel pairs per thread (two pixels each): the constant-bank table operands of a wavelength are
// shared by all of them.
#ifndef SPKB_PRINT_PAIRS
#define SPKB_PRINT_PAIRS 1
#endif
constexpr uint32_t kPairs = SPKB_PRINT_PAIRS;

__device__ __forceinline__ float2 dup(const F32Pair& p) { return make_float2(p.x, p.y); }

// R_k for NP pairs of pixels: sum over l of 2^(e(l)) w_k(l), ascending l. Each table pair, read once per
// wavelength, serves every pair of pixels. Every kPolyEvery-th wavelength takes 2^e from the FMA-pipe
// polynomial (the loop is unrolled, so the choice is made at compile time).
template <int NP>
__device__ __forceinline__ void spectral(const SpectralPairs& t, const float2 (&d)[NP][3], float2 (&r)[NP][3]) {
#pragma unroll
    for (int i = 0; i < NP; ++i) r[i][0] = r[i][1] = r[i][2] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int l = 0; l < SPKB_NL; ++l) {
        const float2 e0 = dup(t.e[3 * l]), e1 = dup(t.e[3 * l + 1]), e2 = dup(t.e[3 * l + 2]);
        const float2 w0 = dup(t.w[3 * l]), w1 = dup(t.w[3 * l + 1]), w2 = dup(t.w[3 * l + 2]);
        const bool poly = kPolyEvery > 0 && l % kPolyEvery == kPolyEvery - 1;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
            const float2 e = __ffma2_rn(d[i][2], e2, __ffma2_rn(d[i][1], e1, __fmul2_rn(d[i][0], e0)));
            const float2 T = poly ? exp2_poly2(e) : make_float2(ex2_ftz(e.x), ex2_ftz(e.y));
            r[i][0] = __ffma2_rn(T, w0, r[i][0]);
            r[i][1] = __ffma2_rn(T, w1, r[i][1]);
            r[i][2] = __ffma2_rn(T, w2, r[i][2]);
        }
    }
}

// Pixels p0 .. p0 + 2 kPairs - 1 of one frame (those below n): the spectral integrals on kPairs packed
// pairs, the rest one pixel after the other.
// enl and scan: the two integrals' tables (a.enl and a.scan, or tables every frame of a batch shares)
__device__ __forceinline__ void print_group(const PrintArgs& a, const SpectralPairs& enl, const SpectralPairs& scan,
                                            const float* __restrict__ neg, float* __restrict__ rgb, uint32_t p0,
                                            uint32_t n) {
    constexpr int NP = kPairs;
    float2 d[NP][3];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        const float* s0 = neg + 3 * size_t(min(p0 + 2 * i, n - 1));
        const float* s1 = neg + 3 * size_t(min(p0 + 2 * i + 1, n - 1));
#pragma unroll
        for (int c = 0; c < 3; ++c) d[i][c] = make_float2(s0[c], s1[c]);
    }
    float2 r[NP][3];
    if (a.printed) {
        spectral<NP>(enl, d, r);
#pragma unroll
        for (int i = 0; i < NP; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                d[i][c] = make_float2(print_density(a, c, r[i][c].x), print_density(a, c, r[i][c].y));
    }
    spectral<NP>(scan, d, r);
#pragma unroll 1
    for (uint32_t k = 0; k < uint32_t(2 * NP); ++k) {
        if (p0 + k >= n) break;
        const uint32_t i = k / 2u;
        const bool hi = (k & 1u) != 0u;
        float x = 0.0f, y = 0.0f, z = 0.0f;
#pragma unroll
        for (int j = 0; j < NP; ++j)
            if (uint32_t(j) == i) {
                x = hi ? r[j][0].y : r[j][0].x;
                y = hi ? r[j][1].y : r[j][1].x;
                z = hi ? r[j][2].y : r[j][2].x;
            }
        x = fmaxf(x, 0.0f) + kTiny;
        y = fmaxf(y, 0.0f) + kTiny;
        z = fmaxf(z, 0.0f) + kTiny;
        apply_levels(a, x, y, z);
        add_glare(a, size_t(p0 + k), x, y, z);
        float rr, g, b;
        mat_apply(a.to_rgb, x, y, z, rr, g, b);
        gamut(a, rr, g, b);
        float* o = rgb + 3 * size_t(p0 + k);
        o[0] = rr;
        o[1] = g;
        o[2] = b;
    }
}

__global__ void __launch_bounds__(kPrintThreads) k_print(const float* __restrict__ neg, float* __restrict__ rgb,
                                                         const __grid_constant__ PrintArgs a) {
    const uint32_t p0 = 2 * kPairs * (blockIdx.x * blockDim.x + threadIdx.x);
    if (p0 >= a.n) return;
    print_group(a, a.enl, a.scan, neg, rgb, p0, a.n);
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
        for (uint32_t p0 = first + 2 * kPairs * threadIdx.x; p0 < min(first + item_px, sa.n);
             p0 += 2 * kPairs * blockDim.x)
            print_group(sa, sa.enl, sa.scan, s_neg, s_rgb, p0, sa.n);
    }
}

// The same with spectral tables that every frame shares (same stocks and filters: the print exposure,
// the planes and the sizes differ), passed in the kernel's parameters so that the unrolled integrals read
// them from the constant bank as k_print does; the per-frame arguments are staged as above (their copy of
// the tables goes unread).
struct SharedSpectra {
    SpectralPairs enl, scan;
};

__global__ void __launch_bounds__(kPrintThreads) k_print_batch_shared(const BatchPrintFrame* __restrict__ frames,
                                                                      const uint32_t* __restrict__ item_frame,
                                                                      const uint32_t* __restrict__ item_first,
                                                                      uint32_t n_items, uint32_t item_px,
                                                                      const __grid_constant__ SharedSpectra t) {
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
        for (uint32_t p0 = first + 2 * kPairs * threadIdx.x; p0 < min(first + item_px, sa.n);
             p0 += 2 * kPairs * blockDim.x)
            print_group(sa, t.enl, t.scan, s_neg, s_rgb, p0, sa.n);
    }
}

}  // namespace

void print(const float* neg, float* rgb, const PrintArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    const uint32_t threads = (a.n + 2 * kPairs - 1) / (2 * kPairs);
    Probe p("print", s);
    k_print<<<(threads + kPrintThreads - 1) / kPrintThreads, kPrintThreads, 0, s>>>(neg, rgb, a);
}

void print_batch(const BatchPrintFrame* frames, const uint32_t* item_frame, const uint32_t* item_first,
                 uint32_t n_items, uint32_t item_px, uint32_t ctas, const SpectralPairs* enl,
                 const SpectralPairs* scan, cudaStream_t s) {
    if (n_items == 0) return;
    Probe p("print_batch", s);
    if (enl && scan) {
        SharedSpectra t;
        t.enl = *enl;
        t.scan = *scan;
        k_print_batch_shared<<<ctas, kPrintThreads, 0, s>>>(frames, item_frame, item_first, n_items, item_px, t);
        return;
    }
    k_print_batch<<<ctas, kPrintThreads, 0, s>>>(frames, item_frame, item_first, n_items, item_px);
}

}  // namespace spkb::dev
