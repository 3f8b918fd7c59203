// Interval search on an ascending binary32 axis, shared by the develop and print kernels (the
// reference's clamped bisection, kernels/film.metal:84-101 and kernels/print.metal:201-232).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"

namespace spkb::dev {
namespace {

// The interval j of v on an ascending axis x[i * stride], i < K: the largest j with x[j] <= v, for v in
// (x[0], x[K-1]); 0 for a NaN v. By a direct index corrected by one step when the host checked the axis
// (AxisGrid), else by bisection; both give the same j.
__device__ __forceinline__ uint32_t axis_index(const float* __restrict__ x, uint32_t stride, uint32_t K,
                                               const AxisGrid& g, float v) {
    if (g.active) {
        int j = int((v - g.x0) * g.s);
        j = min(max(j, 0), int(K) - 2);
        if (__ldg(x + size_t(j) * stride) > v) --j;
        else if (__ldg(x + size_t(j + 1) * stride) <= v) ++j;
        return uint32_t(j);
    }
    uint32_t lo = 0, hi = K;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (__ldg(x + size_t(mid) * stride) <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo == 0 ? 0 : lo - 1;
}

}  // namespace
}  // namespace spkb::dev
