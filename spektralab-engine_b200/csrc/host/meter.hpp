// The auto-exposure meter (reference src/film/meter.cpp): its statistics on the device (csrc/cuda/meter.cu),
// the seven EV values formed from them on the host in binary64.
#pragma once

#include <string_view>

#include "device.hpp"
#include "params.hpp"
#include "resources.hpp"

namespace spkb {

constexpr uint32_t kMeterLongEdge = 1600;  // the meter image's long edge (reference src/session/tiers.hpp)

struct MeterValues {
    double center_weighted = 0.0, average = 0.0, median = 0.0;
    double balanced = 0.0, center = 0.0, protect_highlights = 0.0, protect_shadows = 0.0;
    double ev(std::string_view method) const;
};

// The meter of a meter image (the frame downscaled to 1600 px): decode and geometry as the develop does
// them, then the statistics of its luminance under the input space's RGB -> XYZ row Y.
MeterValues meter(Pool& pool, cudaStream_t s, const Plane& meter_image, const ParamSet& p, const ColourSpace& input);

}  // namespace spkb
