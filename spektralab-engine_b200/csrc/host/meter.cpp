// The auto-exposure meter's host side: the ranks of the order statistics, one device pass of statistics,
// and the seven EV values in binary64 by the reference's formulas (src/film/meter.cpp:45-120).
#include "meter.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../cuda/launch.hpp"
#include "status.hpp"
#include "tiers.hpp"

namespace spkb {

namespace {

constexpr double kMid = 0.184, kFloor = 0.184 / 4096.0;

// -log2(e), 0 when not finite
double legacy_ev(double e) {
    const double ev = -std::log2(e);
    return std::isfinite(ev) ? ev : 0.0;
}
double clampd(double v, double lo, double hi) { return std::min(std::max(v, lo), hi); }

}  // namespace

double MeterValues::ev(std::string_view m) const {
    if (m == "center_weighted") return center_weighted;
    if (m == "average") return average;
    if (m == "median") return median;
    if (m == "balanced") return balanced;
    if (m == "center") return center;
    if (m == "protect_highlights") return protect_highlights;
    if (m == "protect_shadows") return protect_shadows;
    fail_internal("unknown auto-exposure method '" + std::string(m) + "'");
}

MeterValues meter(Pool& pool, cudaStream_t s, const Plane& meter_image, const ParamSet& p, const ColourSpace& input) {
    MeterValues mv;
    const Plane img = prepare_source(pool, s, meter_image, p, p.b(P::input_cctf_decoding), uint32_t(input.cctf));
    const uint64_t n = img.pixels();
    if (n == 0) return mv;
    DevBuffer key = pool.acquire(n * sizeof(uint64_t));
    DevBuffer partial = pool.acquire(dev::meter_partial_doubles() * sizeof(double));
    DevBuffer sel = pool.acquire(sizeof(MeterSelect));
    DevBuffer outb = pool.acquire(sizeof(MeterOut));
    MeterSelect init{};
    init.rank[kMeterMedLo] = (n % 2) ? n / 2 : n / 2 - 1;
    init.rank[kMeterMedHi] = n / 2;
    init.rank[kMeterP10] = 10 * (n - 1) / 1000;
    init.rank[kMeterP50] = 50 * (n - 1) / 1000;
    init.rank[kMeterP990] = 990 * (n - 1) / 1000;
    init.rank[kMeterP995] = 995 * (n - 1) / 1000;
    cuda_check(cudaMemcpyAsync(sel.ptr(), &init, sizeof init, cudaMemcpyHostToDevice, s), "meter set-up");
    MeterArgs a{};
    a.rgb = img.data();
    a.w = img.w;
    a.h = img.h;
    a.n = n;
    a.m0 = input.rgb_to_xyz[3];
    a.m1 = input.rgb_to_xyz[4];
    a.m2 = input.rgb_to_xyz[5];
    a.key = key.as<uint64_t>();
    a.partial = partial.as<double>();
    a.sel = sel.as<MeterSelect>();
    a.out = outb.as<MeterOut>();
    dev::meter_stats(a, s);
    MeterOut o{};
    cuda_check(cudaMemcpyAsync(&o, outb.ptr(), sizeof o, cudaMemcpyDeviceToHost, s), "meter result");
    cuda_check(cudaStreamSynchronize(s), "meter");

    const double sy = o.sums[0], swy = o.sums[1], sw = o.sums[2];
    const double sl = o.sums[3], swl = o.sums[4], sw2 = o.sums[5], cnt = o.sums[6];
    // the y-percentiles are the Y order statistics through std::max(Y, floor) (a NaN stays NaN)
    auto ymax = [](double v) { return v < kFloor ? kFloor : v; };
    mv.average = legacy_ev((sy / double(n)) / kMid);
    const double med = (n % 2) ? o.select[kMeterMedHi] : (o.select[kMeterMedLo] + o.select[kMeterMedHi]) / 2.0;
    mv.median = legacy_ev(med / kMid);
    mv.center_weighted = legacy_ev((swy / sw) / kMid);
    mv.balanced = -std::log2(std::exp(sl / cnt) / kMid);
    mv.center = -std::log2(std::exp(swl / sw2) / kMid);
    mv.protect_highlights =
        clampd(std::log2(kMid * std::pow(2.0, 2.5) / ymax(o.select[kMeterP995])), mv.balanced - 3.0, mv.balanced);
    mv.protect_shadows =
        clampd(std::log2(kMid * std::pow(2.0, -3.5) / ymax(o.select[kMeterP50])), mv.balanced, mv.balanced + 2.0);
    return mv;
}

}  // namespace spkb
