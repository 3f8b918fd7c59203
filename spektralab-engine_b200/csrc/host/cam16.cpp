// CAM16 and CAM16-UCS in binary64 for the print's gamut compression (the model of Li, Li, Wang, Zu, Luo,
// Cui, Melgosa, Brill and Pointer, "Comprehensive color solutions: CAM16, CAT16, and CAM16-UCS", Color
// Research and Application 42 (2017)), under the viewing conditions the reference uses (L_A 64 cd/m^2,
// Y_b 20, average surround; reference src/print/cam16.cpp:41-174):
//   * the viewing constants of a white point;
//   * the forward model to J, C, h, M and the UCS coordinates J', M';
//   * the UCS inverse from (J', a', b'), solved for a and b along the larger of sin h and cos h;
//   * C_max(J', h), the largest M' whose inverse stays inside an RGB cube, by bisection.
// The expressions keep the reference's bracketing so that the narrowed constants and table match it bit for
// bit; the decomposition into the model's named steps is this file's.
#include <algorithm>
#include <cmath>

#include "setup.hpp"

namespace spkb {

namespace {

constexpr Mat3 kM16 = {0.401288, 0.650173, -0.051461, -0.250268, 1.204414, 0.045854, -0.002079, 0.048952, 0.953127};
constexpr double kUcsC1 = 0.007, kUcsC2 = 0.0228;  // CAM16-UCS: J' = 1.7 J / (1 + c1 J), M' = ln(1 + c2 M) / c2

double sign_of(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }

// the post-adaptation non-linearity of one cone response (already scaled by D_rgb)
double compress_response(double v, double F_L) {
    const double f = std::pow((F_L * std::fabs(v)) / 100.0, 0.42);
    return ((400.0 * sign_of(v)) * f) / (27.13 + f) + 0.1;
}
// its inverse, from a post-adaptation value back to the D_rgb-scaled cone response
double expand_response(double v_adapted, double F_L) {
    const double v = v_adapted - 0.1;
    const double mag = std::fabs(v);
    const double base = (27.13 * mag) / (400.0 - mag);
    const double grown = sign_of(base) * std::pow(std::fabs(base), 1.0 / 0.42);
    return ((100.0 / F_L) * sign_of(v)) * grown;
}

struct Adapted {
    double r, g, b;
};
// D_rgb-scaled, compressed cone responses of XYZ (Y = 100 scale)
Adapted adapt(const Cam16Constants& k, const Vec3& xyz100) {
    const Vec3 lms = mat3_apply(k.m16, xyz100);
    return {compress_response(k.D_rgb[0] * lms[0], k.F_L), compress_response(k.D_rgb[1] * lms[1], k.F_L),
            compress_response(k.D_rgb[2] * lms[2], k.F_L)};
}
// the achromatic response A
double achromatic(const Adapted& q, double N_bb) { return (((2.0 * q.r + q.g) + q.b / 20.0) - 0.305) * N_bb; }
// the eccentricity factor e_t of hue angle h (radians)
double eccentricity(double h) { return 0.25 * (std::cos(h + 2.0) + 3.8); }
// the chroma's dependence on the background, (1.64 - 0.29^n)^0.73
double background_gain(const Cam16Constants& k) { return std::pow(1.64 - std::pow(0.29, k.n), 0.73); }
// the common factor of t: (50000 / 13) N_c N_cb e_t
double hue_factor(const Cam16Constants& k, double et) { return (((50000.0 / 13.0) * k.N_c) * k.N_cb) * et; }

// the largest value in [lo, hi] for which inside() holds, by `steps` bisections (inside(lo) assumed)
template <class F>
double bisect_largest(double lo, double hi, int steps, F inside) {
    for (int s = 0; s < steps; ++s) {
        const double mid = (lo + hi) / 2.0;
        if (inside(mid)) lo = mid;
        else hi = mid;
    }
    return lo;
}

}  // namespace

Cam16Constants cam16_constants(const std::array<double, 2>& wp) {
    Cam16Constants k;
    k.m16 = kM16;
    // luminance adaptation
    k.n = k.Y_b / k.Y_w;
    k.k = 1.0 / (5.0 * k.L_A + 1.0);
    const double k4 = k.k * k.k * k.k * k.k;
    const double five_la = 5.0 * k.L_A;
    k.F_L = (0.2 * k4) * five_la + (0.1 * ((1.0 - k4) * (1.0 - k4))) * std::cbrt(five_la);
    k.N_bb = 0.725 * std::pow(1.0 / k.n, 0.2);
    k.N_cb = k.N_bb;
    k.z = 1.48 + std::sqrt(k.n);
    // degree of adaptation, clipped to [0, 1]
    const double degree = k.F * (1.0 - (1.0 / 3.6) * std::exp((-k.L_A - 42.0) / 92.0));
    k.D = std::min(std::max(degree, 0.0), 1.0);
    // the white's cone responses and the von Kries gains
    const Vec3 white = xy_to_XYZ(wp);
    const Vec3 white100 = {100.0 * white[0], 100.0 * white[1], 100.0 * white[2]};
    k.rgb_w = mat3_apply(k.m16, white100);
    for (size_t i = 0; i < 3; ++i) k.D_rgb[i] = (k.D * k.Y_w) / k.rgb_w[i] + 1.0 - k.D;
    k.A_w = achromatic(adapt(k, white100), k.N_bb);
    k.m16_inv = mat3_inverse(k.m16);
    k.J_white = cam16_forward(k, white).Jp;
    return k;
}

Cam16Forward cam16_forward(const Cam16Constants& k, const Vec3& xyz) {
    const Adapted q = adapt(k, {100.0 * xyz[0], 100.0 * xyz[1], 100.0 * xyz[2]});
    // opponent dimensions and hue
    const double a = (q.r - (12.0 * q.g) / 11.0) + q.b / 11.0;
    const double b = ((q.r + q.g) - 2.0 * q.b) / 9.0;
    Cam16Forward f{};
    f.h = std::atan2(b, a);
    // lightness
    const double ratio = achromatic(q, k.N_bb) / k.A_w;
    f.J = (100.0 * sign_of(ratio)) * std::pow(std::fabs(ratio), k.c * k.z);
    // chroma and colourfulness
    const double den = (q.r + q.g) + (21.0 * q.b) / 20.0;
    const double t = den != 0.0 ? (hue_factor(k, eccentricity(f.h)) * std::sqrt(a * a + b * b)) / den : 0.0;
    f.C = t > 0.0 ? (std::pow(t, 0.9) * std::sqrt(std::fabs(f.J) / 100.0)) * background_gain(k) : 0.0;
    f.M = f.C * std::pow(k.F_L, 0.25);
    // the uniform colour space's J' and M'
    f.Mp = std::log(1.0 + kUcsC2 * f.M) / kUcsC2;
    f.Jp = (1.7 * f.J) / (1.0 + kUcsC1 * f.J);
    return f;
}

Vec3 cam16_inverse_unguarded(const Cam16Constants& k, double Jp, double ap, double bp) {
    // UCS back to J, M, C and h
    const double Mp = std::sqrt(ap * ap + bp * bp);
    const double h = std::atan2(bp, ap);
    const double M = (std::exp(kUcsC2 * Mp) - 1.0) / kUcsC2;
    const double J = Jp / (1.7 - kUcsC1 * Jp);
    const double C = M / std::pow(k.F_L, 0.25);
    // achromatic response and t
    const double A = (k.A_w * sign_of(J)) * std::pow(std::fabs(J / 100.0), 1.0 / (k.c * k.z));
    const double root_j = std::sqrt(std::fabs(J) / 100.0);
    const double t = (root_j > 0.0 && C > 0.0) ? std::pow(C / (root_j * background_gain(k)), 1.0 / 0.9) : 0.0;
    // opponent a, b from the two linear equations in them, divided by the larger of sin h and cos h
    const double p2 = A / k.N_bb + 0.305;
    constexpr double p3 = 21.0 / 20.0;
    double a = 0.0, b = 0.0;
    if (t != 0.0) {
        const double p1 = hue_factor(k, eccentricity(h)) / t;
        const double sh = std::sin(h), ch = std::cos(h);
        const double num = (p2 * (2.0 + p3)) * (460.0 / 1403.0);
        if (std::fabs(sh) >= std::fabs(ch)) {
            const double p4 = p1 / sh;
            b = num / (((p4 + ((2.0 + p3) * (220.0 / 1403.0)) * (ch / sh)) - 27.0 / 1403.0) + p3 * (6300.0 / 1403.0));
            a = (b * ch) / sh;
        } else {
            const double p5 = p1 / ch;
            a = num / ((p5 + (2.0 + p3) * (220.0 / 1403.0)) - (27.0 / 1403.0 - p3 * (6300.0 / 1403.0)) * (sh / ch));
            b = (a * sh) / ch;
        }
    }
    // post-adaptation responses, expanded and un-scaled, back to XYZ
    const double adapted[3] = {((460.0 * p2 + 451.0 * a) + 288.0 * b) / 1403.0,
                               ((460.0 * p2 - 891.0 * a) - 261.0 * b) / 1403.0,
                               ((460.0 * p2 - 220.0 * a) - 6300.0 * b) / 1403.0};
    Vec3 lms{};
    for (size_t i = 0; i < 3; ++i) lms[i] = expand_response(adapted[i], k.F_L) / k.D_rgb[i];
    const Vec3 xyz100 = mat3_apply(k.m16_inv, lms);
    return {xyz100[0] / 100.0, xyz100[1] / 100.0, xyz100[2] / 100.0};
}

std::vector<double> cam16_cmax_table(const Cam16Constants& k, const Mat3& m_to_rgb) {
    constexpr int kLightness = 64, kHues = 720, kSteps = 18;
    constexpr double kSlack = 1e-6, kCeiling = 150.0;
    std::vector<double> table(size_t(kLightness) * kHues);
#pragma omp parallel for schedule(dynamic, 1)
    for (int row = 0; row < kLightness; ++row) {
        const double Jp = 1.0 + (109.0 * double(row)) / 63.0;  // J' from 1 to 110
        for (int col = 0; col < kHues; ++col) {
            const double h = -M_PI + (2.0 * M_PI * double(col)) / 720.0;
            const double ch = std::cos(h), sh = std::sin(h);
            table[size_t(row) * kHues + size_t(col)] = bisect_largest(0.0, kCeiling, kSteps, [&](double Mp) {
                const Vec3 rgb = mat3_apply(m_to_rgb, cam16_inverse_unguarded(k, Jp, Mp * ch, Mp * sh));
                for (double v : rgb)
                    if (!(v >= -kSlack && v <= 1.0 + kSlack)) return false;
                return true;
            });
        }
    }
    return table;
}

}  // namespace spkb
