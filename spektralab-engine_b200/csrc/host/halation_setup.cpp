// The film's light-scattering set-up in pixels (reference src/fx/halation.cpp:39-62, :104-195, and the
// exponential surrogate of src/fx/gaussian.cpp:55-66): which halation a stock has, and the Gaussian
// mixtures the render blurs with at a given pixel pitch.
//
//   * scatter: the emulsion's own spread, a core Gaussian plus an exponential tail (as three Gaussians),
//     mixed into the exposure by scatter_amount;
//   * halation: light reflected back from the base, either a series of bounces whose sigma grows with the
//     square root of the bounce number (stocks that keep an anti-halation layer), or a four-component
//     fit of the back-reflection profile (the layer removed); mixed in with strength A per channel.
// The floating-point expressions keep the reference's operation order; constants and tables are the
// physical model's.
#include <algorithm>
#include <cmath>

#include "setup.hpp"

namespace spkb {

namespace {

// Per-channel strength of the reflected light by the stock's anti-halation layer.
struct LayerClass {
    const char* tag;
    Vec3 strength;
};
constexpr LayerClass kLayerClasses[] = {
    {"strong", {0.015, 0.005, 0.0}},
    {"weak", {0.08, 0.02, 0.0}},
    {"no", {0.30, 0.03, 0.003}},  // no layer: the back-reflection profile applies
};

// The back-reflection profile as four Gaussians: sigma in units of the base thickness, and weight, per
// channel (the fit's negative weights shape the ring).
constexpr double kRingSigma[4][3] = {{0.184586, 0.178469, 0.170237},
                                     {1.121207, 1.000078, 0.546805},
                                     {1.651048, 1.581389, 0.808738},
                                     {4.677567, 9.448921, 1.340598}};
constexpr double kRingWeight[4][3] = {{+0.041510, +0.106789, +0.202791},
                                      {-0.500000, -0.500000, +0.156578},
                                      {+1.034500, +1.384389, -0.500000},
                                      {+0.423990, +0.008822, +1.140631}};

// An exponential PSF as three Gaussians: weights and sigmas relative to the exponential's scale.
constexpr double kExpWeight[3] = {0.1633, 0.6496, 0.1870};
constexpr double kExpSigma[3] = {0.5360, 1.5236, 2.7684};

constexpr double kMinSigma = 1e-6;

MixtureComponent component(const Vec3& weight, const Vec3& sigma) {
    MixtureComponent m;
    m.weight = weight;
    m.sigma = sigma;
    return m;
}

// the emulsion scatter: the core Gaussian and the tail's surrogate, or nothing
void add_scatter(const HalationParams& h, double pitch_um, HalationPlan& plan) {
    Vec3 core{}, tail{};
    bool sized = false;
    for (size_t c = 0; c < 3; ++c) {
        core[c] = h.scatter_core_um[c] * h.scatter_scale / pitch_um;
        tail[c] = h.scatter_tail_um[c] * h.scatter_scale / pitch_um;
        sized = sized || core[c] != 0.0 || tail[c] != 0.0;
    }
    if (!(h.scatter_amount > 0.0) || !sized) return;
    Vec3 core_w{}, core_s{}, tail_s{};
    for (size_t c = 0; c < 3; ++c) {
        core_w[c] = 1.0 - h.scatter_tail_weight[c];
        core_s[c] = std::max(core[c], kMinSigma);
        tail_s[c] = std::max(tail[c], kMinSigma);
    }
    plan.scatter = true;
    plan.scatter_comps.push_back(component(core_w, core_s));
    for (const MixtureComponent& m : exponential_surrogate(h.scatter_tail_weight, tail_s)) plan.scatter_comps.push_back(m);
    const double keep = 1.0 - h.scatter_amount;
    plan.scatter_a = {keep, keep, keep};
    plan.scatter_b = {h.scatter_amount, h.scatter_amount, h.scatter_amount};
}

// bounces k = 1..n with weights decay^(k - 1) normalised to one and sigma s sqrt(k)
void add_bounces(const HalationParams& h, const Vec3& first_px, HalationPlan& plan) {
    double norm = 0.0;
    for (int k = 1; k <= h.bounces; ++k) norm += std::pow(h.bounce_decay, double(k - 1));
    for (int k = 1; k <= h.bounces; ++k) {
        const double wk = std::pow(h.bounce_decay, double(k - 1)) / norm;
        Vec3 s{};
        for (size_t c = 0; c < 3; ++c) s[c] = std::max(first_px[c] * std::sqrt(double(k)), kMinSigma);
        plan.bounce_comps.push_back(component({wk, wk, wk}, s));
    }
    plan.bounce = true;
}

// the back-reflection ring for a base of thickness base_px
void add_ring(double base_px, HalationPlan& plan) {
    for (int k = 0; k < 4; ++k) {
        Vec3 w{}, s{};
        for (size_t c = 0; c < 3; ++c) {
            w[c] = kRingWeight[k][c];
            s[c] = std::max(kRingSigma[k][c] * base_px, kMinSigma);
        }
        plan.bounce_comps.push_back(component(w, s));
    }
    plan.bounce = true;
}

}  // namespace

HalationParams resolve_halation(const Profile& film, const ParamSet& p) {
    HalationParams h;
    h.active = p.b(P::halation_active);
    h.amount = p.f(P::halation_amount);
    h.scatter_amount = p.f(P::halation_scatter_amount);
    h.headroom_ev = p.f(P::halation_headroom_ev);
    if (film.support != "film") return h;  // prints and digital sources keep the defaults
    const std::string tag = p.b(P::antihalation_removed) ? std::string("no") : film.antihalation;
    const LayerClass* cls = nullptr;
    for (const LayerClass& lc : kLayerClasses)
        if (tag == lc.tag) cls = &lc;
    if (!cls || (film.use != "still" && film.use != "cine")) return h;
    const double first = film.use == "cine" ? 50.0 : 65.0;  // the first bounce's sigma in micrometres
    h.first_sigma_um = {first, first, first};
    h.strength = cls->strength;
    h.back_reflection = std::string(cls->tag) == "no";
    return h;
}

std::array<MixtureComponent, 3> exponential_surrogate(const Vec3& weight, const Vec3& lambda_px) {
    std::array<MixtureComponent, 3> out{};
    for (size_t i = 0; i < 3; ++i)
        for (size_t c = 0; c < 3; ++c) {
            out[i].weight[c] = weight[c] * kExpWeight[i];
            out[i].sigma[c] = kExpSigma[i] * lambda_px[c];
        }
    return out;
}

HalationPlan halation_plan(const HalationParams& h, double pitch_um) {
    HalationPlan plan;
    if (!h.active) return plan;
    add_scatter(h, pitch_um, plan);
    // the strength per channel is formed in binary32, as the reference's kernel arguments are
    Vec3 A{};
    bool strong = false;
    const float amount32 = f32(h.amount);
    for (size_t c = 0; c < 3; ++c) {
        A[c] = double(f32(h.strength[c]) * amount32);
        strong = strong || A[c] > 0.0;
    }
    const double grow = std::sqrt(std::max(h.amount, 0.0));  // sigmas grow with the square root of the amount
    if (h.back_reflection) {
        const double base_px = h.base_thickness_um * h.halation_scale * grow / pitch_um;
        if (strong && base_px > 0.0) add_ring(base_px, plan);
    } else {
        Vec3 first{};
        bool sized = false;
        for (size_t c = 0; c < 3; ++c) {
            first[c] = h.first_sigma_um[c] * h.halation_scale * grow / pitch_um;
            sized = sized || first[c] > 0.0;
        }
        if (h.bounces >= 1 && strong && sized) add_bounces(h, first, plan);
    }
    if (plan.bounce)
        for (size_t c = 0; c < 3; ++c) {
            plan.mix_a[c] = h.renormalise ? 1.0 / (1.0 + A[c]) : 1.0;
            plan.mix_b[c] = h.renormalise ? A[c] / (1.0 + A[c]) : A[c];
        }
    return plan;
}

}  // namespace spkb
