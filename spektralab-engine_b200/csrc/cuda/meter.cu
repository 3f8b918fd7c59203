// The auto-exposure meter's statistics on the device (reference src/film/meter.cpp:45-120, which does them
// in binary64 on the CPU with two full sorts of the meter image).
//
// Here nothing is sorted: the order statistics (the median and the 1, 5, 99 and 99.5 % points) come from
// one multi-query radix select over the pixels' binary64 luminances mapped to ordered 64-bit keys, eight
// passes of 8-bit digits, each pass a histogram launch and a one-block resolve launch. The luminance, the
// centre weight and the log sums are the reference's binary64 formulas, each operation rounded on its
// own (no contraction). Sums are taken per block in a fixed order and then over the blocks in one thread,
// so repeated meters give the same bits; they differ from the reference's sequential sums only in the
// last bits. The host reads back 13 doubles and forms the seven EV values.
#include <cuda_runtime.h>
#include <stdint.h>

#include "launch.hpp"

namespace spkb::dev {

namespace {

constexpr int kBlocks = 512, kThreads = 256;
constexpr double kFloor = 0.184 / 4096.0, kTwoS2 = 2.0 * (0.2 * 0.2);

__device__ __forceinline__ double luma(const MeterArgs& a, size_t k) {
    const float* p = a.rgb + 3 * k;
    return __dadd_rn(__dadd_rn(__dmul_rn(a.m0, double(p[0])), __dmul_rn(a.m1, double(p[1]))),
                     __dmul_rn(a.m2, double(p[2])));
}

// exp(-(x^2 + y^2) / (2 0.2^2)), x and y the pixel's offsets from the centre in units of the long edge
__device__ __forceinline__ double centre_weight(const MeterArgs& a, size_t k) {
    const uint32_t col = uint32_t(k % a.w), row = uint32_t(k / a.w);
    const double M = double(a.w > a.h ? a.w : a.h);
    const double x = __dmul_rn(__dsub_rn(__ddiv_rn(double(col), double(a.w)), 0.5), __ddiv_rn(double(a.w), M));
    const double y = __dmul_rn(__dsub_rn(__ddiv_rn(double(row), double(a.h)), 0.5), __ddiv_rn(double(a.h), M));
    return exp(__ddiv_rn(-__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), kTwoS2));
}

// ascending order of the doubles, NaN last
__device__ __forceinline__ uint64_t order_key(double v) {
    if (isnan(v)) return ~0ull;
    const uint64_t b = uint64_t(__double_as_longlong(v));
    return (b >> 63) ? ~b : (b | (1ull << 63));
}
__device__ __forceinline__ double key_value(uint64_t k) {
    if (k == ~0ull) return __longlong_as_double(0x7ff8000000000000ll);
    return __longlong_as_double((long long)((k >> 63) ? (k & ~(1ull << 63)) : ~k));
}

// block sum of v in thread order: a shared-memory tree, the same for every launch
__device__ __forceinline__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (int(threadIdx.x) < s) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kThreads) k_meter_luma(const __grid_constant__ MeterArgs a) {
    __shared__ double sh[kThreads];
    double sy = 0.0, swy = 0.0, sw = 0.0;
    for (size_t k = size_t(blockIdx.x) * kThreads + threadIdx.x; k < a.n; k += size_t(kBlocks) * kThreads) {
        const double Y = luma(a, k);
        const double w = centre_weight(a, k);
        a.key[k] = order_key(Y);
        sy = __dadd_rn(sy, Y);
        swy = __dadd_rn(swy, __dmul_rn(w, Y));
        sw = __dadd_rn(sw, w);
    }
    sy = block_sum(sy, sh);
    swy = block_sum(swy, sh);
    sw = block_sum(sw, sh);
    if (threadIdx.x == 0) {
        a.partial[0 * kBlocks + blockIdx.x] = sy;
        a.partial[1 * kBlocks + blockIdx.x] = swy;
        a.partial[2 * kBlocks + blockIdx.x] = sw;
    }
}

// One digit of the radix select: per query, the histogram of digit `shift` over the keys that match the
// query's prefix so far.
__global__ void __launch_bounds__(kThreads) k_meter_hist(const __grid_constant__ MeterArgs a, int shift) {
    __shared__ uint32_t hist[kMeterQueries][256];
    for (int i = threadIdx.x; i < kMeterQueries * 256; i += kThreads) (&hist[0][0])[i] = 0;
    __syncthreads();
    uint64_t prefix[kMeterQueries], mask[kMeterQueries];
#pragma unroll
    for (int q = 0; q < kMeterQueries; ++q) {
        prefix[q] = a.sel->prefix[q];
        mask[q] = a.sel->mask[q];
    }
    for (size_t k = size_t(blockIdx.x) * kThreads + threadIdx.x; k < a.n; k += size_t(kBlocks) * kThreads) {
        const uint64_t key = a.key[k];
        const uint32_t d = uint32_t(key >> shift) & 255u;
#pragma unroll
        for (int q = 0; q < kMeterQueries; ++q)
            if ((key & mask[q]) == prefix[q]) atomicAdd(&hist[q][d], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kMeterQueries * 256; i += kThreads) {
        const uint32_t c = (&hist[0][0])[i];
        if (c) atomicAdd(&a.sel->hist[0][0] + i, c);
    }
}

// The digit that holds each query's rank; the histogram is cleared for the next pass. After the last
// digit the prefix is the key itself and the selected value is stored.
__global__ void k_meter_resolve(const __grid_constant__ MeterArgs a, int shift) {
    const int q = threadIdx.x;
    if (q >= kMeterQueries) return;
    MeterSelect& s = *a.sel;
    uint64_t below = 0;
    int d = 0;
    for (; d < 255; ++d) {
        const uint64_t c = s.hist[q][d];
        if (below + c > s.rank[q]) break;
        below += c;
    }
    s.rank[q] -= below;
    s.prefix[q] |= uint64_t(d) << shift;
    s.mask[q] |= 255ull << shift;
    for (int i = 0; i < 256; ++i) s.hist[q][i] = 0;
    if (shift == 0) s.value[q] = key_value(s.prefix[q]);
}

// The intent meters' sums over the pixels inside [P(1 %), P(99 %)] of y = max(Y, mid / 4096).
__global__ void __launch_bounds__(kThreads) k_meter_intent(const __grid_constant__ MeterArgs a) {
    __shared__ double sh[kThreads];
    // y's order statistics are those of Y through the same max (a NaN stays NaN and then admits nothing)
    const double v1 = a.sel->value[kMeterP10], v99 = a.sel->value[kMeterP990];
    const double p1 = v1 < kFloor ? kFloor : v1, p99 = v99 < kFloor ? kFloor : v99;
    double sl = 0.0, swl = 0.0, sw = 0.0, cnt = 0.0;
    for (size_t k = size_t(blockIdx.x) * kThreads + threadIdx.x; k < a.n; k += size_t(kBlocks) * kThreads) {
        const double Y = luma(a, k);
        const double y = Y < kFloor ? kFloor : Y;  // std::max(Y, floor): NaN stays NaN
        if (!(y >= p1 && y <= p99)) continue;
        const double l = log(y);
        const double w = centre_weight(a, k);
        sl = __dadd_rn(sl, l);
        swl = __dadd_rn(swl, __dmul_rn(w, l));
        sw = __dadd_rn(sw, w);
        cnt += 1.0;
    }
    sl = block_sum(sl, sh);
    swl = block_sum(swl, sh);
    sw = block_sum(sw, sh);
    cnt = block_sum(cnt, sh);
    if (threadIdx.x == 0) {
        a.partial[3 * kBlocks + blockIdx.x] = sl;
        a.partial[4 * kBlocks + blockIdx.x] = swl;
        a.partial[5 * kBlocks + blockIdx.x] = sw;
        a.partial[6 * kBlocks + blockIdx.x] = cnt;
    }
}

// The block partials summed in block order, and the selected values, into the result.
__global__ void k_meter_finish(const __grid_constant__ MeterArgs a) {
    const int i = threadIdx.x;
    if (i < 7) {
        double s = 0.0;
        for (int b = 0; b < kBlocks; ++b) s = __dadd_rn(s, a.partial[i * kBlocks + b]);
        a.out->sums[i] = s;
    } else if (i < 7 + kMeterQueries) {
        a.out->select[i - 7] = a.sel->value[i - 7];
    }
}

}  // namespace

size_t meter_partial_doubles() { return size_t(7) * kBlocks; }

void meter_stats(const MeterArgs& a, cudaStream_t s) {
    {
        Probe p("meter_luma", s);
        k_meter_luma<<<kBlocks, kThreads, 0, s>>>(a);
    }
    for (int shift = 56; shift >= 0; shift -= 8) {
        {
            Probe p("meter_hist", s);
            k_meter_hist<<<kBlocks, kThreads, 0, s>>>(a, shift);
        }
        Probe p("meter_resolve", s);
        k_meter_resolve<<<1, 32, 0, s>>>(a, shift);
    }
    {
        Probe p("meter_intent", s);
        k_meter_intent<<<kBlocks, kThreads, 0, s>>>(a);
    }
    Probe p("meter_finish", s);
    k_meter_finish<<<1, 32, 0, s>>>(a);
}

}  // namespace spkb::dev
