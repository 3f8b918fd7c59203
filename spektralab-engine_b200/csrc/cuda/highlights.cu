// The film side's two highlight stages between the exposure and the halation (reference
// src/film/develop.cpp:32-62 and :155-168, kernels/film.metal:229-239, kernels/fx_halation.metal:13-39):
// the highlight boost and the back-reflection halation's headroom. Both take the frame's maximum, which
// k_plane_max forms exactly (a max does not depend on order) as an order-preserving integer with one
// atomicMax per block; the headroom kernel reads it from device memory, the boost's host reads it back.
#include <cuda_runtime.h>
#include <stdint.h>

#include "launch.hpp"

namespace spkb::dev {

namespace {

// floats in ascending order as unsigned integers (NaN never stored: the max skips it)
__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b >> 31) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t u) { return __uint_as_float((u >> 31) ? (u & 0x7fffffffu) : ~u); }

__global__ void k_plane_max_init(uint32_t* out) { *out = ordered(-INFINITY); }

__global__ void k_plane_max(const float* __restrict__ p, size_t n, uint32_t* out) {
    float m = -INFINITY;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float v = p[i];
        if (v > m) m = v;  // NaN is skipped, as in the reference's host loop
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31u) == 0) atomicMax(out, ordered(m));
}

__global__ void k_plane_max_read(const uint32_t* in, float* out) { *out = unordered(*in); }

__device__ __forceinline__ float smooth01(float t) {
    const float u = fminf(fmaxf(t, 0.0f), 1.0f);
    return __fmul_rn(__fmul_rn(u, u), __fsub_rn(3.0f, __fmul_rn(2.0f, u)));
}

// all channels times 2^(headroom_ev s1 s2), s1 and s2 smooth steps of the pixel's log2 max channel
// against the frame's clip and mid grey; skipped when the clip is not a positive finite number
__global__ void k_headroom(float* p, uint32_t n, const uint32_t* clip_ord, float headroom_ev) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float clip = unordered(*clip_ord);
    if (!(clip > 0.0f) || !isfinite(clip)) return;
    float* v = p + 3 * size_t(i);
    const float m = fmaxf(fmaxf(v[0], v[1]), v[2]);
    float g = 1.0f;
    if (m > 0.0f) {
        const float lm = log2f(m);
        const float s1 = smooth01(__fdiv_rn(__fadd_rn(__fsub_rn(lm, log2f(clip)), 1.0f), 0.75f));
        const float s2 = smooth01(__fsub_rn(__fsub_rn(lm, log2f(0.184f)), 1.5f));
        g = exp2f(__fmul_rn(__fmul_rn(headroom_ev, s1), s2));
    }
    v[0] = __fmul_rn(v[0], g);
    v[1] = __fmul_rn(v[1], g);
    v[2] = __fmul_rn(v[2], g);
}

// v > x0: v + k (exp(z) - z - 1), z = a (v - x0) r
__global__ void k_boost(float* p, size_t n, float x0, float r, float a, float k) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = p[i];
    if (!(v > x0)) return;
    const float z = __fmul_rn(a, __fmul_rn(__fsub_rn(v, x0), r));
    const float w = __fsub_rn(__fsub_rn(expf(z), z), 1.0f);
    p[i] = __fadd_rn(v, __fmul_rn(k, w));
}

}  // namespace

void plane_max(const float* p, size_t n, uint32_t* out_ordered, cudaStream_t s) {
    k_plane_max_init<<<1, 1, 0, s>>>(out_ordered);
    Probe pr("plane_max", s);
    k_plane_max<<<592, 256, 0, s>>>(p, n, out_ordered);
}

void plane_max_value(const uint32_t* ordered_max, float* out, cudaStream_t s) {
    k_plane_max_read<<<1, 1, 0, s>>>(ordered_max, out);
}

void headroom(float* p, uint32_t pixels, const uint32_t* clip_ordered, float headroom_ev, cudaStream_t s) {
    Probe pr("headroom", s);
    k_headroom<<<(pixels + 255) / 256, 256, 0, s>>>(p, pixels, clip_ordered, headroom_ev);
}

void boost(float* p, size_t n, float x0, float r, float a, float k, cudaStream_t s) {
    Probe pr("boost", s);
    k_boost<<<unsigned((n + 255) / 256), 256, 0, s>>>(p, n, x0, r, a, k);
}

}  // namespace spkb::dev
