// The film side's binary64 set-up (reference src/film/setup.cpp:25-95, :353-419, src/fx/grain.cpp:66-152,
// src/fx/gaussian.cpp:19-53): the input transform, the spectral upsampling table (upsampling.cpp), the
// density-curve lookup tables, the DIR couplers' matrix and pre-inverted curves, the grain's layer tables and
// per-pitch constants, and the blur kernels' coefficients. Narrowed once to binary32 for the kernels; the
// binary64 expressions keep the reference's operation order (the narrowed values are pinned bit for bit
// against it), the decomposition and names are this file's.
#include <cmath>

#include "setup.hpp"
#include "status.hpp"

namespace spkb {

// =============================== Gaussian blurs ==================================================

Branch blur_branch(double sigma) {
    if (!(sigma > 0.0)) return Branch::Identity;
    return sigma < 3.0 ? Branch::Fir : Branch::Iir;
}

int fir_radius(double sigma) { return sigma > 0.0 ? int(std::floor(3.0 * sigma + 0.5)) : 0; }

std::vector<double> gaussian_kernel(double sigma, double truncate) {
    const int radius = sigma > 0.0 ? int(std::floor(truncate * sigma + 0.5)) : 0;
    if (radius == 0) return {1.0};
    std::vector<double> taps;
    taps.reserve(size_t(2 * radius + 1));
    double total = 0.0;
    for (int k = -radius; k <= radius; ++k) {
        const double u = double(k) / sigma;
        taps.push_back(std::exp(-0.5 * u * u));
        total += taps.back();
    }
    for (double& t : taps) t /= total;
    return taps;
}

// Young and van Vliet, "Recursive implementation of the Gaussian filter", Signal Processing 44 (1995): the
// scale q of sigma (two regimes), the cubic's coefficients b0..b3, and the normalised feedback weights.
IirCoefficients iir_coefficients(double sigma) {
    const double q = sigma >= 2.5 ? 0.98711 * sigma - 0.96330 : 3.97156 - 4.14554 * std::sqrt(1.0 - 0.26891 * sigma);
    const double q2 = q * q, q3 = q2 * q;
    const double b0 = ((1.57825 + 2.44413 * q) + 1.4281 * q2) + 0.422205 * q3;
    const double b1 = (2.44413 * q + 2.85619 * q2) + 1.26661 * q3;
    const double b2 = -(1.4281 * q2 + 1.26661 * q3);
    const double b3 = 0.422205 * q3;
    IirCoefficients c;
    c.B1 = b1 / b0;
    c.B2 = b2 / b0;
    c.B3 = b3 / b0;
    c.B = 1.0 - ((b1 + b2) + b3) / b0;
    return c;
}

IirCoefficients iir_coefficients_dsigma(double sigma) {
    // q(sigma) and dq/dsigma in the regime iir_coefficients uses
    double q, dq;
    if (sigma >= 2.5) {
        q = 0.98711 * sigma - 0.96330;
        dq = 0.98711;
    } else {
        const double r = std::sqrt(1.0 - 0.26891 * sigma);
        q = 3.97156 - 4.14554 * r;
        dq = 4.14554 * 0.26891 / (2.0 * r);
    }
    const double q2 = q * q, q3 = q2 * q;
    const double b0 = ((1.57825 + 2.44413 * q) + 1.4281 * q2) + 0.422205 * q3;
    const double b1 = (2.44413 * q + 2.85619 * q2) + 1.26661 * q3;
    const double b2 = -(1.4281 * q2 + 1.26661 * q3);
    const double b3 = 0.422205 * q3;
    const double d0 = 2.44413 + 2.0 * 1.4281 * q + 3.0 * 0.422205 * q2;  // db_i / dq
    const double d1 = 2.44413 + 2.0 * 2.85619 * q + 3.0 * 1.26661 * q2;
    const double d2 = -(2.0 * 1.4281 * q + 3.0 * 1.26661 * q2);
    const double d3 = 3.0 * 0.422205 * q2;
    auto ratio = [&](double b, double d) { return (d * b0 - b * d0) / (b0 * b0) * dq; };  // d(b / b0) / dsigma
    IirCoefficients c;
    c.B1 = ratio(b1, d1);
    c.B2 = ratio(b2, d2);
    c.B3 = ratio(b3, d3);
    c.B = -((c.B1 + c.B2) + c.B3);
    return c;
}

std::vector<double> gaussian_kernel_dsigma(double sigma, double truncate) {
    const std::vector<double> w = gaussian_kernel(sigma, truncate);
    const int radius = int(w.size() / 2);
    double second = 0.0;  // sum_j w_j j^2
    for (int k = -radius; k <= radius; ++k) second += w[size_t(k + radius)] * double(k) * double(k);
    const double s3 = sigma * sigma * sigma;
    std::vector<double> d(w.size());
    for (int k = -radius; k <= radius; ++k)
        d[size_t(k + radius)] = w[size_t(k + radius)] * (double(k) * double(k) - second) / s3;
    return d;
}

// =============================== grain ===========================================================

namespace {

// the grain model's constants: a silver particle's area (um^2), per-channel and per-sub-layer particle
// scales, the final blur in pixels, the dye-cloud and micro-structure blurs in micrometres
constexpr double kParticleArea = 0.2;
constexpr double kChannelScale[3] = {1.6, 1.6, 3.2};
constexpr double kSublayerScale[3] = {2.0, 1.0, 0.5};
constexpr double kFinalBlurPx = 0.65;
constexpr double kDyeBlurUm = 1.0;
constexpr double kMicroBlurUm = 0.2;
constexpr double kMicroSigmaNm = 30.0;

// the layer tables of a stock with per-sub-layer density curves: each sub-layer's share of the channel's
// density range, its saturation density, and the curve lookup (the normalised curve, sign-flipped for a
// positive stock, its reciprocal steps and the K x 3 x 3 sub-layer curves) in binary32
std::shared_ptr<GrainSetup> grain_layers(const Profile& film, const ParamSet& p) {
    auto g = std::make_shared<GrainSetup>();
    g->active = p.b(P::grain_active);
    g->sublayers = p.b(P::grain_sublayers_active);
    g->amount = p.f(P::grain_amount);
    g->positive = film.positive();
    const bool has_layers = !film.layers.empty();
    if (g->active && g->sublayers && !has_layers)
        fail_user("grain sub-layers: film stock '" + film.id + "' has no per-layer density curves (density_curves_layers)");
    for (size_t c = 0; c < 3; ++c) g->simple_d[c] = film.dmax[c] + kGrainDmin[c];
    if (!has_layers) return g;
    const size_t K = film.K();
    g->K = uint32_t(K);
    for (size_t c = 0; c < 3; ++c) {
        double top[3];
        for (size_t l = 0; l < 3; ++l) top[l] = nanmax_strided(film.layers.data() + l * 3 + c, K, 9);
        const double range = (top[0] + top[1]) + top[2];
        for (size_t l = 0; l < 3; ++l) {
            g->f[l][c] = top[l] / range;
            g->dmin[l][c] = g->f[l][c] * kGrainDmin[c];
            g->sat_d[l][c] = top[l] + g->dmin[l][c];
        }
    }
    std::vector<double> curve(K * 3);
    for (size_t k = 0; k < K; ++k)
        for (size_t c = 0; c < 3; ++c) curve[k * 3 + c] = g->positive ? -film.normalized(k, c) : film.normalized(k, c);
    g->axis.resize(K * 3);
    g->inv.assign(K * 3, 0.0f);
    for (size_t i = 0; i < K * 3; ++i) g->axis[i] = f32(curve[i]);
    for (size_t k = 0; k + 1 < K; ++k)
        for (size_t c = 0; c < 3; ++c) {
            const double step = curve[(k + 1) * 3 + c] - curve[k * 3 + c];
            g->inv[k * 3 + c] = step == 0.0 ? 0.0f : f32(1.0 / step);
        }
    g->layers.resize(K * 9);
    for (size_t i = 0; i < K * 9; ++i) g->layers[i] = f32(film.layers[i]);
    return g;
}

}  // namespace

GrainConstants grain_constants(const GrainSetup& g, double pitch_um) {
    GrainConstants k;
    k.active = g.active && g.amount > 0.0;
    k.sublayers = g.sublayers;
    const double area = pitch_um * pitch_um;  // a pixel's area in um^2
    if (!g.sublayers) {
        for (size_t c = 0; c < 3; ++c) {
            k.count[0][c] = area / (kParticleArea * kChannelScale[c]);
            k.sat_d[0][c] = g.simple_d[c];
        }
        k.final_blur = kFinalBlurPx > 0.4 ? kFinalBlurPx : 0.0;
        return k;
    }
    for (size_t l = 0; l < 3; ++l)
        for (size_t c = 0; c < 3; ++c) {
            const double particles = (area * g.f[l][c]) / ((kParticleArea * kChannelScale[c]) * kSublayerScale[l]);
            k.count[l][c] = particles;
            k.sat_d[l][c] = g.sat_d[l][c];
            k.dmin_l[l][c] = g.dmin[l][c];
            const double dye = kDyeBlurUm * std::sqrt(g.sat_d[l][c] / particles);  // a dye cloud's spread
            k.sigma_dye[l][c] = dye > 0.4 ? dye : 0.0;
            k.dye = k.dye || k.sigma_dye[l][c] > 0.0;
        }
    k.micro_sigma = kMicroSigmaNm * 0.001 / pitch_um;
    k.micro = k.micro_sigma > 0.05;
    k.micro_blur = kMicroBlurUm / pitch_um;
    k.final_blur = kFinalBlurPx;
    return k;
}

// =============================== film set-up =====================================================

namespace {

// DIR coupler gains of a stock, by donor layer (rows) and receiving layer (columns): the self-inhibition on
// the diagonal, the cross terms off it
struct CouplerGains {
    const char* stock;  // nullptr: the class default below
    double self_r, self_g, self_b, r_to_g, r_to_b, g_to_r, g_to_b, b_to_r, b_to_g;
    Mat3 matrix() const { return {self_r, r_to_g, r_to_b, g_to_r, self_g, g_to_b, b_to_r, b_to_g, self_b}; }
};
constexpr CouplerGains kCouplerStocks[] = {
    {"fujifilm_velvia_100", 0.108, 0.072, 0.054, 0.108, 0.054, 0.072, 0.054, 0.054, 0.054},
    {"fujifilm_provia_100f", 0.156, 0.104, 0.078, 0.156, 0.078, 0.104, 0.078, 0.078, 0.078},
};
constexpr CouplerGains kCouplerPositive = {nullptr, 0.12, 0.08, 0.06, 0.12, 0.06, 0.08, 0.06, 0.06, 0.06};
constexpr CouplerGains kCouplerNegative = {nullptr, 0.336, 0.319, 0.273, 0.353, 0.302, 0.154, 0.353, 0.168, 0.226};

Mat3 coupler_matrix(const Profile& film, double amount) {
    const CouplerGains* g = film.positive() ? &kCouplerPositive : &kCouplerNegative;
    for (const CouplerGains& s : kCouplerStocks)
        if (film.id == s.stock) g = &s;
    const Mat3 base = g->matrix();
    Mat3 m{};
    for (size_t i = 0; i < 9; ++i) m[i] = amount * base[i];
    return m;
}

// the curve lookup: x = log10 exposure / gamma, 1 / dx, and the normalised curves (channel-major)
void curve_tables(const Profile& film, double gamma, FilmSetup& s) {
    const size_t K = film.K();
    const std::vector<double>& le = film.log_exposure;
    s.K = uint32_t(K);
    s.cx.resize(K);
    s.cinv.assign(K, 0.0f);
    s.cy.resize(3 * K);
    for (size_t k = 0; k < K; ++k) {
        s.cx[k] = f32(le[k] / gamma);
        if (k + 1 < K) {
            const double dx = le[k + 1] / gamma - le[k] / gamma;
            s.cinv[k] = dx == 0.0 ? 0.0f : f32(1.0 / dx);
        }
        for (size_t c = 0; c < 3; ++c) s.cy[c * K + k] = f32(film.normalized(k, c));
    }
}

// the couplers' pre-inverted curves: with couplers a layer's density D_m develops at log exposure
// x - sum_c s_c M[c][m] (s_c the donor's density, or its distance from D_max for a positive stock), so the
// curve y0_m is the stock's curve read back at that shifted axis, sampled on the plain axis
void pre_inverted_curves(const Profile& film, const Mat3& m, FilmSetup& s) {
    const size_t K = film.K();
    const std::vector<double>& le = film.log_exposure;
    s.cy0.resize(3 * K);
    s.cy0_64.resize(3 * K);
    std::vector<double> shifted(K), density(K);
    for (size_t recv = 0; recv < 3; ++recv) {
        for (size_t k = 0; k < K; ++k) {
            double inhibition = 0.0;
            for (size_t donor = 0; donor < 3; ++donor) {
                const double sd = s.positive ? film.dmax[donor] - film.normalized(k, donor) : film.normalized(k, donor);
                inhibition += sd * m[3 * donor + recv];
            }
            shifted[k] = le[k] - inhibition;
            density[k] = film.normalized(k, recv);
        }
        for (size_t k = 0; k < K; ++k) {
            s.cy0_64[recv * K + k] = interp(le[k], shifted, density);
            s.cy0[recv * K + k] = f32(s.cy0_64[recv * K + k]);
        }
    }
}

}  // namespace

std::shared_ptr<FilmSetup> build_film_setup(const ParamSet& p, std::shared_ptr<const Profile> film_ptr,
                                            const Resources& res) {
    const Profile& film = *film_ptr;
    const Blob& blob = res.blob();
    auto s = std::make_shared<FilmSetup>();
    s->params = p;
    s->profile = film_ptr;
    s->positive = film.positive();
    // the input transform: the input space's RGB to XYZ, adapted (CAT16) to the film's reference illuminant
    const std::string& space = p.s(P::input_color_space);
    const std::optional<ColourSpace> in = colour_space(blob, space);
    if (!in) fail_user("input_color_space: the resources have no colour space called '" + space + "'");
    s->input_space = *in;
    s->decode = p.b(P::input_cctf_decoding);
    const std::optional<Spectrum> light = illuminant(blob, film.reference_illuminant);
    if (!light)
        fail_user("film stock '" + film.id + "': its reference_illuminant '" + film.reference_illuminant +
                  "' is not in the resources");
    s->illuminant_xy = chromaticity(blob, *light);
    const std::optional<Mat3> cat16 = cat_matrix(blob, "CAT16");
    if (!cat16) fail_user("input transform: the resources have no colour/cat/CAT16 matrix");
    const std::optional<Mat3> adapt = von_kries(s->input_space.whitepoint, s->illuminant_xy, *cat16, Guard::Source);
    s->input_matrix = adapt ? mat3_mul(*adapt, s->input_space.rgb_to_xyz) : s->input_space.rgb_to_xyz;
    for (size_t i = 0; i < 9; ++i) s->input_matrix_f32[i] = f32(s->input_matrix[i]);
    // the layers' spectral sensitivities (undefined bins count as zero) and the upsampling table
    std::array<double, 243> sens{};
    for (size_t b = 0; b < 81; ++b)
        for (size_t c = 0; c < 3; ++c) {
            const double v = std::pow(10.0, film.log_sensitivity(b, c));
            sens[3 * b + c] = std::isnan(v) ? 0.0 : v;
        }
    s->table64 = spectral_upsampling_table(blob, sens, film.window, *light, &s->L);
    s->table32.resize(s->table64.size());
    for (size_t i = 0; i < s->table64.size(); ++i) s->table32[i] = f32(s->table64[i]);
    s->halation = resolve_halation(film, p);
    if (p.b(P::grain_active)) s->grain = grain_layers(film, p);
    // the density curves and the couplers
    if (film.K() < 2) fail_user("film stock '" + film.id + "': its log_exposure axis needs two points or more");
    curve_tables(film, p.f(P::density_curve_gamma), *s);
    s->couplers = p.b(P::dir_couplers_active);
    s->coupler_m = coupler_matrix(film, p.f(P::dir_couplers_amount));
    for (size_t i = 0; i < 9; ++i) s->coupler_m_f32[i] = f32(s->coupler_m[i]);
    for (size_t c = 0; c < 3; ++c) {
        s->dmax[c] = film.dmax[c];
        s->dmax_f32[c] = f32(film.dmax[c]);
    }
    pre_inverted_curves(film, s->coupler_m, *s);
    return s;
}

// =============================== CAM16-UCS tables per output space ===============================

std::shared_ptr<const Cam16Tables> Cam16Cache::get(const Resources& res, const std::string& space) {
    std::lock_guard<std::mutex> g(m_);
    if (auto it = by_space_.find(space); it != by_space_.end()) return it->second;
    if (!cctf_of(space)) fail_user("gamut compression: '" + space + "' is not one of the known colour spaces");
    const std::optional<ColourSpace> cs = colour_space(res.blob(), space);
    if (!cs) fail_user("gamut compression: the resources have no matrices or white point for '" + space + "'");
    if (cs->whitepoint[1] == 0.0) fail_user("gamut compression: the white point of '" + space + "' has y = 0");
    auto t = std::make_shared<Cam16Tables>();
    t->space = space;
    t->k = cam16_constants(cs->whitepoint);
    t->m_to_xyz = cs->rgb_to_xyz;
    t->m_to_rgb = cs->xyz_to_rgb;
    t->cmax64 = cam16_cmax_table(t->k, cs->xyz_to_rgb);
    t->cmax32.resize(t->cmax64.size());
    for (size_t i = 0; i < t->cmax64.size(); ++i) t->cmax32[i] = f32(t->cmax64[i]);
    by_space_[space] = t;
    return t;
}

}  // namespace spkb
