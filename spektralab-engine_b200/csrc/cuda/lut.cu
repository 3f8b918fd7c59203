// The print-preview table render (reference kernels/print.metal:368-407, src/print/run.cpp:190-223): the
// negative's densities index a trilinear S x S x S x 3 table (interpolated along k, then j, then i), and
// the result is encoded to RGBA16 in the table's own encoding. Each operation is rounded on its own, as in
// the reference's CPU build. The table (59 KB at S = 17) stays in L1/L2; reads go through the read-only path.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"
#include "encode.cuh"
#include "launch.hpp"

namespace spkb::dev {

namespace {

__device__ __forceinline__ float lerp_rn(float a, float b, float f) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, f)), __fmul_rn(b, f));
}

__global__ void k_print_lut(const float* __restrict__ neg, uint16_t* __restrict__ out,
                            const __grid_constant__ PrintLutArgs a) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = 3 * (size_t(y) * a.w + x);
    const uint32_t S = a.size;
    uint32_t i0[3], i1[3];
    float f[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float u = __fmul_rn(fminf(fmaxf(__fmul_rn(__fsub_rn(neg[i + c], a.lo[c]), a.s[c]), 0.0f), 1.0f),
                                  float(S - 1));
        const float fl = floorf(u);
        i0[c] = uint32_t(fl);
        f[c] = __fsub_rn(u, fl);
        i1[c] = min(i0[c] + 1, S - 1);
    }
    uint16_t* o = out + 4 * (size_t(y) * a.stride + x);
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float c[2][2];
#pragma unroll
        for (int di = 0; di < 2; ++di)
#pragma unroll
            for (int dj = 0; dj < 2; ++dj) {
                const size_t base = (size_t(di ? i1[0] : i0[0]) * S + (dj ? i1[1] : i0[1])) * S;
                c[di][dj] = lerp_rn(__ldg(a.lut + (base + i0[2]) * 3 + ch), __ldg(a.lut + (base + i1[2]) * 3 + ch), f[2]);
            }
        const float v = __fadd_rn(__fmul_rn(lerp_rn(c[0][0], c[0][1], f[1]), __fsub_rn(1.0f, f[0])),
                                  __fmul_rn(lerp_rn(c[1][0], c[1][1], f[1]), f[0]));
        o[ch] = encode16(v);
    }
    o[3] = 65535;
}

}  // namespace

void print_lut(const float* neg, uint16_t* out, const PrintLutArgs& a, cudaStream_t s) {
    const dim3 b(32, 8), g((a.w + 31) / 32, (a.h + 7) / 8);
    Probe p("print_lut", s);
    k_print_lut<<<g, b, 0, s>>>(neg, out, a);
}

}  // namespace spkb::dev
