// The steps before the film path: the tier downscale of the frame (reference src/session/tiers.cpp) and
// the input decode + geometry (reference src/film/geometry.cpp), with their binary64 set-up on the host.
#pragma once

#include <cstdint>
#include <vector>

#include "device.hpp"
#include "params.hpp"

namespace spkb {

constexpr uint32_t kPreviewLongEdge = 3400;  // the preview tier (reference src/session/tiers.hpp:24)

struct Size2 {
    uint32_t w = 0, h = 0;
};

// The tier's image size for a frame of w x h and a target long edge (0: the frame's own size):
// floor of each side scaled by long_edge / max(w, h), at least 1 (reference src/session/tiers.cpp:50-57).
Size2 downscale_size(uint32_t w, uint32_t h, uint32_t long_edge);

// The per-axis prefilter taps, gaussian with sigma = max(0, (n / m - 1) / 2) truncated at 4 sigma,
// binary64 normalised then narrowed ({1}: no prefilter on the axis).
std::vector<float> tier_axis_taps(uint32_t n, uint32_t m);

// The per-axis bilinear source indices (i0, i1 per output) and weights t, in exact integers: the source
// coordinate (o + 1/2) n / m - 1/2 mirrored into [0, n - 1].
struct TierAxisSamples {
    std::vector<uint32_t> idx;
    std::vector<float> t;
};
TierAxisSamples tier_axis_samples(uint32_t n, uint32_t m);

// The tier image of `src` at target long edge L on the device (src itself when no downscale applies).
Plane downscale(Pool& pool, cudaStream_t s, const Plane& src, uint32_t long_edge);

bool geometry_identity(const ParamSet& p);
// The develop's plane size for a tier image of w x h: the geometry's output size, or w x h.
Size2 prepared_size(const ParamSet& p, uint32_t w, uint32_t h);

// The decode + geometry stage of the develop (reference src/film/geometry.cpp:45-107, :159-200): `src`
// when neither applies, else a new plane of the geometry's output size (the rounded crop, its sides
// exchanged by an odd quarter turn).
Plane prepare_source(Pool& pool, cudaStream_t s, const Plane& src, const ParamSet& p, bool decode, uint32_t cctf_mode);

}  // namespace spkb
