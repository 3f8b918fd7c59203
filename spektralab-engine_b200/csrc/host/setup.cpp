#include "setup.hpp"

#include <cmath>
#include <cstring>
#include <limits>

#include "status.hpp"

namespace spkb {

// =============================== Gaussian machinery ===============================================

Branch blur_branch(double sigma) {
    if (!(sigma > 0.0)) return Branch::Identity;
    return sigma < 3.0 ? Branch::Fir : Branch::Iir;
}

int fir_radius(double sigma) {
    if (!(sigma > 0.0)) return 0;
    return int(std::floor(3.0 * sigma + 0.5));
}

// w_k = exp(-0.5 (k / sigma)^2), k = -r..r, divided by their sum accumulated in ascending k
// (reference src/util/numeric.cpp gaussian_kernel).
std::vector<double> gaussian_kernel(double sigma, double truncate) {
    const int r = sigma > 0.0 ? int(std::floor(truncate * sigma + 0.5)) : 0;
    if (r == 0) return {1.0};
    std::vector<double> w(size_t(2 * r + 1));
    double sum = 0.0;
    for (int k = -r; k <= r; ++k) {
        const double t = double(k) / sigma;
        const double e = std::exp(-0.5 * t * t);
        w[size_t(k + r)] = e;
        sum += e;
    }
    for (double& e : w) e /= sum;
    return w;
}

// Young and van Vliet, "Recursive implementation of the Gaussian filter", Signal Processing 44 (1995):
// q from sigma, then b0..b3 and the normalised B, B1, B2, B3 (B + B1 + B2 + B3 = 1).
IirCoefficients iir_coefficients(double sigma) {
    double q;
    if (sigma >= 2.5) q = 0.98711 * sigma - 0.96330;
    else q = 3.97156 - 4.14554 * std::sqrt(1.0 - 0.26891 * sigma);
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

// =============================== halation ========================================================

HalationParams resolve_halation(const Profile& film, const ParamSet& p) {
    HalationParams h;
    h.active = p.b(P::halation_active);
    h.amount = p.f(P::halation_amount);
    h.scatter_amount = p.f(P::halation_scatter_amount);
    h.headroom_ev = p.f(P::halation_headroom_ev);
    if (film.support != "film") return h;
    const std::string tag = p.b(P::antihalation_removed) ? std::string("no") : film.antihalation;
    Vec3 strength;
    if (tag == "strong") strength = {0.015, 0.005, 0.0};
    else if (tag == "weak") strength = {0.08, 0.02, 0.0};
    else if (tag == "no") strength = {0.30, 0.03, 0.003};
    else return h;
    if (film.use != "still" && film.use != "cine") return h;
    const double s = film.use == "cine" ? 50.0 : 65.0;
    h.first_sigma_um = {s, s, s};
    h.strength = strength;
    h.back_reflection = tag == "no";
    return h;
}

// An exponential PSF as three Gaussians (reference src/fx/gaussian.cpp:55-66).
std::array<MixtureComponent, 3> exponential_surrogate(const Vec3& weight, const Vec3& lambda_px) {
    static constexpr double kA[3] = {0.1633, 0.6496, 0.1870};
    static constexpr double kR[3] = {0.5360, 1.5236, 2.7684};
    std::array<MixtureComponent, 3> out{};
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) {
            out[size_t(i)].weight[size_t(c)] = weight[size_t(c)] * kA[i];
            out[size_t(i)].sigma[size_t(c)] = kR[i] * lambda_px[size_t(c)];
        }
    return out;
}

HalationPlan halation_plan(const HalationParams& h, double p) {
    HalationPlan pl;
    if (!h.active) return pl;
    Vec3 core{}, lam{};
    bool any_size = false;
    for (size_t c = 0; c < 3; ++c) {
        core[c] = h.scatter_core_um[c] * h.scatter_scale / p;
        lam[c] = h.scatter_tail_um[c] * h.scatter_scale / p;
        any_size = any_size || core[c] != 0.0 || lam[c] != 0.0;
    }
    if (h.scatter_amount > 0.0 && any_size) {
        pl.scatter = true;
        MixtureComponent c0;
        Vec3 lam1{};
        for (size_t c = 0; c < 3; ++c) {
            c0.weight[c] = 1.0 - h.scatter_tail_weight[c];
            c0.sigma[c] = std::max(core[c], 1e-6);
            lam1[c] = std::max(lam[c], 1e-6);
        }
        pl.scatter_comps.push_back(c0);
        for (const MixtureComponent& m : exponential_surrogate(h.scatter_tail_weight, lam1)) pl.scatter_comps.push_back(m);
        const double sa = h.scatter_amount;
        pl.scatter_a = {1.0 - sa, 1.0 - sa, 1.0 - sa};
        pl.scatter_b = {sa, sa, sa};
    }
    Vec3 A{};
    bool any_a = false;
    const float famount = f32(h.amount);
    for (size_t c = 0; c < 3; ++c) {
        const float prod = f32(h.strength[c]) * famount;
        A[c] = double(prod);
        any_a = any_a || A[c] > 0.0;
    }
    const double rho = std::sqrt(std::max(h.amount, 0.0));
    if (!h.back_reflection) {
        Vec3 sh{};
        bool any_sigma = false;
        for (size_t c = 0; c < 3; ++c) {
            sh[c] = h.first_sigma_um[c] * h.halation_scale * rho / p;
            any_sigma = any_sigma || sh[c] > 0.0;
        }
        if (h.bounces >= 1 && any_a && any_sigma) {
            double total = 0.0;
            for (int j = 1; j <= h.bounces; ++j) total += std::pow(h.bounce_decay, double(j - 1));
            for (int k = 1; k <= h.bounces; ++k) {
                MixtureComponent m;
                const double wk = std::pow(h.bounce_decay, double(k - 1)) / total;
                for (size_t c = 0; c < 3; ++c) {
                    m.weight[c] = wk;
                    m.sigma[c] = std::max(sh[c] * std::sqrt(double(k)), 1e-6);
                }
                pl.bounce_comps.push_back(m);
            }
            pl.bounce = true;
        }
    } else {
        static constexpr double kS[4][3] = {{0.184586, 0.178469, 0.170237},
                                            {1.121207, 1.000078, 0.546805},
                                            {1.651048, 1.581389, 0.808738},
                                            {4.677567, 9.448921, 1.340598}};
        static constexpr double kW[4][3] = {{+0.041510, +0.106789, +0.202791},
                                            {-0.500000, -0.500000, +0.156578},
                                            {+1.034500, +1.384389, -0.500000},
                                            {+0.423990, +0.008822, +1.140631}};
        const double dp = h.base_thickness_um * h.halation_scale * rho / p;
        if (any_a && dp > 0.0) {
            for (int k = 0; k < 4; ++k) {
                MixtureComponent m;
                for (size_t c = 0; c < 3; ++c) {
                    m.weight[c] = kW[k][c];
                    m.sigma[c] = std::max(kS[k][c] * dp, 1e-6);
                }
                pl.bounce_comps.push_back(m);
            }
            pl.bounce = true;
        }
    }
    if (pl.bounce) {
        for (size_t c = 0; c < 3; ++c) {
            if (h.renormalise) {
                pl.mix_a[c] = 1.0 / (1.0 + A[c]);
                pl.mix_b[c] = A[c] / (1.0 + A[c]);
            } else {
                pl.mix_a[c] = 1.0;
                pl.mix_b[c] = A[c];
            }
        }
    }
    return pl;
}

// =============================== grain ===========================================================

namespace {
constexpr double kParticleArea = 0.2;
constexpr double kChannelScale[3] = {1.6, 1.6, 3.2};
constexpr double kSublayerScale[3] = {2.0, 1.0, 0.5};
constexpr double kFinalBlurPx = 0.65;
constexpr double kDyeBlurUm = 1.0;
constexpr double kMicroBlurUm = 0.2;
constexpr double kMicroSigmaNm = 30.0;
constexpr int kSimpleSublayers = 1;

std::shared_ptr<GrainSetup> build_grain_setup(const Profile& film, const ParamSet& p) {
    auto g = std::make_shared<GrainSetup>();
    g->active = p.b(P::grain_active);
    g->sublayers = p.b(P::grain_sublayers_active);
    g->amount = p.f(P::grain_amount);
    g->positive = film.positive();
    const size_t K = film.K();
    const bool has_layers = !film.layers.empty();
    if (g->active && g->sublayers && !has_layers)
        fail_user("film profile '" + film.id + "' has no density_curves_layers, which grain sublayers need");
    for (size_t c = 0; c < 3; ++c) g->simple_d[c] = film.dmax[c] + kGrainDmin[c];
    if (!has_layers) return g;
    g->K = uint32_t(K);
    double dmax_raw[3][3];
    for (size_t l = 0; l < 3; ++l)
        for (size_t c = 0; c < 3; ++c) dmax_raw[l][c] = nanmax_strided(film.layers.data() + l * 3 + c, K, 9);
    for (size_t c = 0; c < 3; ++c) {
        const double T = (dmax_raw[0][c] + dmax_raw[1][c]) + dmax_raw[2][c];
        for (size_t l = 0; l < 3; ++l) {
            g->f[l][c] = dmax_raw[l][c] / T;
            g->dmin[l][c] = g->f[l][c] * kGrainDmin[c];
            g->sat_d[l][c] = dmax_raw[l][c] + g->dmin[l][c];
        }
    }
    std::vector<double> a(K * 3);
    for (size_t k = 0; k < K; ++k)
        for (size_t c = 0; c < 3; ++c) {
            const double v = film.normalized(k, c);
            a[k * 3 + c] = g->positive ? -v : v;
        }
    g->axis.resize(K * 3);
    g->inv.assign(K * 3, 0.0f);
    for (size_t i = 0; i < K * 3; ++i) g->axis[i] = f32(a[i]);
    for (size_t k = 0; k + 1 < K; ++k)
        for (size_t c = 0; c < 3; ++c) {
            const double step = a[(k + 1) * 3 + c] - a[k * 3 + c];
            g->inv[k * 3 + c] = step == 0.0 ? 0.0f : f32(1.0 / step);
        }
    g->layers.resize(K * 9);
    for (size_t i = 0; i < K * 9; ++i) g->layers[i] = f32(film.layers[i]);
    return g;
}
}  // namespace

GrainConstants grain_constants(const GrainSetup& g, double p) {
    GrainConstants k;
    k.active = g.active && g.amount > 0.0;
    k.sublayers = g.sublayers;
    const double p2 = p * p;
    if (g.sublayers) {
        for (size_t l = 0; l < 3; ++l)
            for (size_t c = 0; c < 3; ++c) {
                const double n = (p2 * g.f[l][c]) / ((kParticleArea * kChannelScale[c]) * kSublayerScale[l]);
                k.count[l][c] = n;
                k.sat_d[l][c] = g.sat_d[l][c];
                k.dmin_l[l][c] = g.dmin[l][c];
                const double s = kDyeBlurUm > 0.0 ? kDyeBlurUm * std::sqrt(g.sat_d[l][c] / n) : 0.0;
                k.sigma_dye[l][c] = s > 0.4 ? s : 0.0;
                k.dye = k.dye || k.sigma_dye[l][c] > 0.0;
            }
        k.micro_sigma = kMicroSigmaNm * 0.001 / p;
        k.micro = k.micro_sigma > 0.05;
        k.micro_blur = kMicroBlurUm / p;
        k.final_blur = kFinalBlurPx;
    } else {
        for (size_t c = 0; c < 3; ++c) {
            double n = p2 / (kParticleArea * kChannelScale[c]);
            if (kSimpleSublayers > 1) n = n / kSimpleSublayers;
            k.count[0][c] = n;
            k.sat_d[0][c] = g.simple_d[c];
        }
        k.final_blur = kFinalBlurPx > 0.4 ? kFinalBlurPx : 0.0;
    }
    return k;
}

// =============================== film set-up =====================================================

namespace {

double clip01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

std::array<double, 2> q_map(double x, double y) {
    const double o = 1.0 - x;
    return {clip01(o * o), clip01(y / std::max(o, 1e-10))};
}

Mat3 coupler_matrix(const Profile& film, double amount) {
    auto make = [](double sr, double sg, double sb, double rg, double rb, double gr, double gb, double br, double bg) {
        return Mat3{sr, rg, rb, gr, sg, gb, br, bg, sb};
    };
    Mat3 g;
    if (film.id == "fujifilm_velvia_100") g = make(0.108, 0.072, 0.054, 0.108, 0.054, 0.072, 0.054, 0.054, 0.054);
    else if (film.id == "fujifilm_provia_100f") g = make(0.156, 0.104, 0.078, 0.156, 0.078, 0.104, 0.078, 0.078, 0.078);
    else if (film.positive()) g = make(0.12, 0.08, 0.06, 0.12, 0.06, 0.08, 0.06, 0.06, 0.06);
    else g = make(0.336, 0.319, 0.273, 0.353, 0.302, 0.154, 0.353, 0.168, 0.226);
    Mat3 m{};
    for (size_t r = 0; r < 3; ++r)
        for (size_t c = 0; c < 3; ++c) m[3 * r + c] = amount * (1.0 * g[3 * r + c]);
    return m;
}

// The spectral-upsampling table T' (reference src/film/setup.cpp:133-257): the film-layer response
// of every chromaticity node's spectrum, then the input gamut compression baked in by a ray cast from
// the illuminant's white to the spectrum locus and a (0, 1, 6) knee on the radius.
std::vector<double> spectral_table(const Blob& blob, const std::array<double, 243>& S, const std::vector<double>& window,
                                   const Spectrum& I, uint32_t* L_out) {
    const BlobEntry* e = blob.find("hanatos/spectra_lut");
    if (!e || e->ndim != 3 || e->dims[0] != e->dims[1] || e->dims[2] != 81 || e->dims[0] < 2)
        fail_user("film set-up: the constants blob has no usable hanatos/spectra_lut (L x L x 81)");
    const uint32_t L = e->dims[0];
    const std::vector<double> spectra = blob.f64("hanatos/spectra_lut");
    *L_out = L;
    std::array<double, 243> W = S;
    if (!window.empty()) {
        if (window.size() != 4) fail_user("film set-up: only the 4-parameter adaptation window is built");
        const double cuv = window[0], suv = window[1], cir = window[2], sir = window[3];
        const double r2 = std::sqrt(2.0);
        std::array<double, 81> om{};
        for (size_t l = 0; l < 81; ++l) {
            const double lam = 380.0 + 5.0 * double(l);
            om[l] = 0.5 * (1.0 + std::erf((lam - cuv) / (suv * r2))) * (0.5 * (1.0 - std::erf((lam - cir) / (sir * r2))));
        }
        for (size_t c = 0; c < 3; ++c) {
            double num = 0.0, den = 0.0;
            for (size_t l = 0; l < 81; ++l) {
                num += S[3 * l + c] * om[l] * I[l];
                den += S[3 * l + c] * I[l];
            }
            const double f = num / den;
            for (size_t l = 0; l < 81; ++l) W[3 * l + c] = S[3 * l + c] * om[l] / f;
        }
    }
    const size_t nodes = size_t(L) * L;
    std::vector<double> T(nodes * 3);
    for (size_t n = 0; n < nodes; ++n) {
        const double* s = spectra.data() + n * 81;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (size_t l = 0; l < 81; ++l) {
            a0 += s[l] * W[3 * l];
            a1 += s[l] * W[3 * l + 1];
            a2 += s[l] * W[3 * l + 2];
        }
        T[3 * n] = a0;
        T[3 * n + 1] = a1;
        T[3 * n + 2] = a2;
    }
    const std::vector<double> cmf = blob.f64("colour/cmfs_1931_2deg");
    if (cmf.size() != 243) fail_user("film set-up: colour/cmfs_1931_2deg must be 81 x 3");
    std::array<double, 2> w{};
    {
        double X = 0, Y = 0, Z = 0;
        for (size_t l = 0; l < 81; ++l) {
            X += I[l] * cmf[3 * l];
            Y += I[l] * cmf[3 * l + 1];
            Z += I[l] * cmf[3 * l + 2];
        }
        const double t = X + Y + Z;
        w = {X / t, Y / t};
    }
    std::vector<std::array<double, 2>> poly;
    for (size_t l = 0; l <= 64; ++l) {
        const double X = cmf[3 * l], Y = cmf[3 * l + 1], Z = cmf[3 * l + 2];
        const double s = std::max(X + Y + Z, 1e-12);
        poly.push_back({X / s, Y / s});
    }
    poly.push_back(poly.front());
    const double last = double(L - 1);
    std::vector<double> Tp(nodes * 3);
    for (uint32_t i = 0; i < L; ++i) {
        for (uint32_t j = 0; j < L; ++j) {
            const double t0 = double(i) / last, t1 = double(j) / last;
            const double sq = std::sqrt(t0);
            const std::array<double, 2> p{1.0 - sq, t1 * sq};
            const double dx = p[0] - w[0], dy = p[1] - w[1];
            const double d = std::sqrt(dx * dx + dy * dy);
            std::array<double, 2> pp = p;
            if (!(d < 1e-9)) {
                const double dm = std::max(d, 1e-12);
                const double ux = dx / dm, uy = dy / dm;
                double beta = std::numeric_limits<double>::infinity();
                for (size_t k = 0; k + 1 < poly.size(); ++k) {
                    const double ex = poly[k + 1][0] - poly[k][0], ey = poly[k + 1][1] - poly[k][1];
                    const double den = ux * ey - uy * ex;
                    if (std::fabs(den) <= 1e-12) continue;
                    const double ox = w[0] - poly[k][0], oy = w[1] - poly[k][1];
                    const double s = (-ox * ey + oy * ex) / den;
                    const double v = (-ox * uy + oy * ux) / den;
                    if (v >= 0.0 && v <= 1.0 && s > 1e-9 && s < beta) beta = s;
                }
                const double r = d / std::max(beta, 1e-12);
                double rp = r;
                if (r > 0.0) {
                    const double z = (r - 0.0) / (1.0 - 0.0);
                    rp = 0.0 + (1.0 - 0.0) * z / std::pow(1.0 + std::pow(z, 6.0), 1.0 / 6.0);
                }
                pp = {w[0] + ux * rp * beta, w[1] + uy * rp * beta};
            }
            const std::array<double, 2> tq = q_map(pp[0], pp[1]);
            auto axis = [&](double tv, uint32_t& a0, uint32_t& a1, double& f) {
                double c = tv * last;
                if (!(c > 0.0)) c = 0.0;
                if (c > last) c = last;
                const double fl = std::floor(c);
                a0 = uint32_t(fl);
                a1 = std::min(a0 + 1, L - 1);
                f = c - fl;
            };
            uint32_t i0, i1, j0, j1;
            double fi, fj;
            axis(tq[0], i0, i1, fi);
            axis(tq[1], j0, j1, fj);
            const double* v00 = &T[3 * (size_t(i0) * L + j0)];
            const double* v01 = &T[3 * (size_t(i0) * L + j1)];
            const double* v10 = &T[3 * (size_t(i1) * L + j0)];
            const double* v11 = &T[3 * (size_t(i1) * L + j1)];
            double* o = &Tp[3 * (size_t(i) * L + j)];
            for (size_t c = 0; c < 3; ++c)
                o[c] = v00[c] * (1.0 - fi) * (1.0 - fj) + v01[c] * (1.0 - fi) * fj + v10[c] * fi * (1.0 - fj) +
                       v11[c] * fi * fj;
        }
    }
    return Tp;
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
    const std::string& space = p.s(P::input_color_space);
    auto cs = colour_space(blob, space);
    if (!cs) fail_user("input_color_space '" + space + "' is not a colour space in the constants blob");
    s->input_space = *cs;
    s->decode = p.b(P::input_cctf_decoding);
    auto I = illuminant(blob, film.reference_illuminant);
    if (!I) fail_user("film '" + film.id + "': unknown reference_illuminant '" + film.reference_illuminant + "'");
    s->illuminant_xy = chromaticity(blob, *I);
    auto cat16 = cat_matrix(blob, "CAT16");
    if (!cat16) fail_user("film set-up: the constants blob has no colour/cat/CAT16");
    auto C = von_kries(s->input_space.whitepoint, s->illuminant_xy, *cat16, Guard::Source);
    s->input_matrix = C ? mat3_mul(*C, s->input_space.rgb_to_xyz) : s->input_space.rgb_to_xyz;
    for (size_t i = 0; i < 9; ++i) s->input_matrix_f32[i] = f32(s->input_matrix[i]);
    std::array<double, 243> sens{};
    for (size_t l = 0; l < 81; ++l)
        for (size_t c = 0; c < 3; ++c) {
            const double v = std::pow(10.0, film.log_sensitivity(l, c));
            sens[3 * l + c] = std::isnan(v) ? 0.0 : v;
        }
    s->table64 = spectral_table(blob, sens, film.window, *I, &s->L);
    s->table32.resize(s->table64.size());
    for (size_t i = 0; i < s->table64.size(); ++i) s->table32[i] = f32(s->table64[i]);
    s->halation = resolve_halation(film, p);
    if (p.b(P::grain_active)) s->grain = build_grain_setup(film, p);

    const size_t K = film.K();
    if (K < 2) fail_user("film '" + film.id + "': log_exposure needs at least 2 points");
    const double gamma = p.f(P::density_curve_gamma);
    const Mat3 m = coupler_matrix(film, p.f(P::dir_couplers_amount));
    s->K = uint32_t(K);
    s->cx.resize(K);
    s->cinv.assign(K, 0.0f);
    s->cy.resize(3 * K);
    s->cy0.resize(3 * K);
    s->cy0_64.resize(3 * K);
    s->couplers = p.b(P::dir_couplers_active);
    s->coupler_m = m;
    for (size_t i = 0; i < 9; ++i) s->coupler_m_f32[i] = f32(m[i]);
    for (size_t c = 0; c < 3; ++c) {
        s->dmax[c] = film.dmax[c];
        s->dmax_f32[c] = f32(film.dmax[c]);
    }
    const std::vector<double>& le = film.log_exposure;
    for (size_t k = 0; k < K; ++k) {
        s->cx[k] = f32(le[k] / gamma);
        if (k + 1 < K) {
            const double d = le[k + 1] / gamma - le[k] / gamma;
            s->cinv[k] = d == 0.0 ? 0.0f : f32(1.0 / d);
        }
        for (size_t c = 0; c < 3; ++c) s->cy[c * K + k] = f32(film.normalized(k, c));
    }
    std::vector<double> xs(K), ys(K);
    for (size_t mm = 0; mm < 3; ++mm) {
        for (size_t k = 0; k < K; ++k) {
            double sum = 0.0;
            for (size_t c = 0; c < 3; ++c) {
                const double sigma = s->positive ? film.dmax[c] - film.normalized(k, c) : film.normalized(k, c);
                sum += sigma * m[3 * c + mm];
            }
            xs[k] = le[k] - sum;
            ys[k] = film.normalized(k, mm);
        }
        for (size_t k = 0; k < K; ++k) {
            s->cy0_64[mm * K + k] = interp(le[k], xs, ys);
            s->cy0[mm * K + k] = f32(s->cy0_64[mm * K + k]);
        }
    }
    return s;
}

// =============================== CAM16-UCS ========================================================

namespace {
double sgn(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }
constexpr Mat3 kM16 = {0.401288, 0.650173, -0.051461, -0.250268, 1.204414, 0.045854, -0.002079, 0.048952, 0.953127};
constexpr Mat3 kM16InvPublished = {1.86206786,  -1.01125463, 0.14918677,  0.38752654, 0.62144744,
                                   -0.00897398, -0.01584150, -0.03412294, 1.04996444};
double post_adapt(double v, double F_L) {
    const double f = std::pow((F_L * std::fabs(v)) / 100.0, 0.42);
    return ((400.0 * sgn(v)) * f) / (27.13 + f) + 0.1;
}
}  // namespace

// Li et al., "Comprehensive color solutions: CAM16, CAT16, and CAM16-UCS", Color Research and
// Application 42 (2017); viewing conditions L_A 64, Y_b 20, average surround.
Cam16Constants cam16_constants(const std::array<double, 2>& wp) {
    Cam16Constants k;
    k.m16 = kM16;
    k.n = k.Y_b / k.Y_w;
    k.k = 1.0 / (5.0 * k.L_A + 1.0);
    const double k4 = k.k * k.k * k.k * k.k;
    const double la5 = 5.0 * k.L_A;
    k.F_L = (0.2 * k4) * la5 + (0.1 * ((1.0 - k4) * (1.0 - k4))) * std::cbrt(la5);
    k.N_bb = 0.725 * std::pow(1.0 / k.n, 0.2);
    k.N_cb = k.N_bb;
    k.z = 1.48 + std::sqrt(k.n);
    const double D = k.F * (1.0 - (1.0 / 3.6) * std::exp((-k.L_A - 42.0) / 92.0));
    k.D = D < 0.0 ? 0.0 : (D > 1.0 ? 1.0 : D);
    const Vec3 xyz = xy_to_XYZ(wp);
    const Vec3 xyz_w = {100.0 * xyz[0], 100.0 * xyz[1], 100.0 * xyz[2]};
    k.rgb_w = mat3_apply(k.m16, xyz_w);
    for (int i = 0; i < 3; ++i) k.D_rgb[i] = (k.D * k.Y_w) / k.rgb_w[i] + 1.0 - k.D;
    const double ra = post_adapt(k.D_rgb[0] * k.rgb_w[0], k.F_L);
    const double ga = post_adapt(k.D_rgb[1] * k.rgb_w[1], k.F_L);
    const double ba = post_adapt(k.D_rgb[2] * k.rgb_w[2], k.F_L);
    k.A_w = (((2.0 * ra + ga) + ba / 20.0) - 0.305) * k.N_bb;
    k.m16_inv = mat3_inverse(k.m16);
    k.J_white = cam16_forward(k, xyz).Jp;
    return k;
}

Cam16Forward cam16_forward(const Cam16Constants& k, const Vec3& xyz) {
    const Vec3 x100 = {100.0 * xyz[0], 100.0 * xyz[1], 100.0 * xyz[2]};
    const Vec3 rgb = mat3_apply(k.m16, x100);
    const double ra = post_adapt(k.D_rgb[0] * rgb[0], k.F_L);
    const double ga = post_adapt(k.D_rgb[1] * rgb[1], k.F_L);
    const double ba = post_adapt(k.D_rgb[2] * rgb[2], k.F_L);
    const double a = (ra - (12.0 * ga) / 11.0) + ba / 11.0;
    const double b = ((ra + ga) - 2.0 * ba) / 9.0;
    Cam16Forward f{};
    f.h = std::atan2(b, a);
    const double et = 0.25 * (std::cos(f.h + 2.0) + 3.8);
    const double A = (((2.0 * ra + ga) + ba / 20.0) - 0.305) * k.N_bb;
    const double ratio = A / k.A_w;
    f.J = (100.0 * sgn(ratio)) * std::pow(std::fabs(ratio), k.c * k.z);
    const double den = (ra + ga) + (21.0 * ba) / 20.0;
    const double t = den != 0.0 ? (((((50000.0 / 13.0) * k.N_c) * k.N_cb) * et) * std::sqrt(a * a + b * b)) / den : 0.0;
    f.C = t > 0.0 ? (std::pow(t, 0.9) * std::sqrt(std::fabs(f.J) / 100.0)) * std::pow(1.64 - std::pow(0.29, k.n), 0.73)
                  : 0.0;
    f.M = f.C * std::pow(k.F_L, 0.25);
    f.Mp = std::log(1.0 + 0.0228 * f.M) / 0.0228;
    f.Jp = (1.7 * f.J) / (1.0 + 0.007 * f.J);
    return f;
}

Vec3 cam16_inverse_unguarded(const Cam16Constants& k, double Jp, double ap, double bp) {
    const double Mp = std::sqrt(ap * ap + bp * bp);
    const double h = std::atan2(bp, ap);
    const double M = (std::exp(0.0228 * Mp) - 1.0) / 0.0228;
    const double J = Jp / (1.7 - 0.007 * Jp);
    const double C = M / std::pow(k.F_L, 0.25);
    const double A = (k.A_w * sgn(J)) * std::pow(std::fabs(J / 100.0), 1.0 / (k.c * k.z));
    const double sq = std::sqrt(std::fabs(J) / 100.0);
    const double t =
        (sq > 0.0 && C > 0.0) ? std::pow(C / (sq * std::pow(1.64 - std::pow(0.29, k.n), 0.73)), 1.0 / 0.9) : 0.0;
    const double et = 0.25 * (std::cos(h + 2.0) + 3.8);
    const double p2 = A / k.N_bb + 0.305;
    const double p3 = 21.0 / 20.0;
    double a = 0.0, b = 0.0;
    if (t != 0.0) {
        const double p1 = ((((50000.0 / 13.0) * k.N_c) * k.N_cb) * et) / t;
        const double sh = std::sin(h), ch = std::cos(h);
        if (std::fabs(sh) >= std::fabs(ch)) {
            const double p4 = p1 / sh;
            b = ((p2 * (2.0 + p3)) * (460.0 / 1403.0)) /
                (((p4 + ((2.0 + p3) * (220.0 / 1403.0)) * (ch / sh)) - 27.0 / 1403.0) + p3 * (6300.0 / 1403.0));
            a = (b * ch) / sh;
        } else {
            const double p5 = p1 / ch;
            a = ((p2 * (2.0 + p3)) * (460.0 / 1403.0)) /
                ((p5 + (2.0 + p3) * (220.0 / 1403.0)) - (27.0 / 1403.0 - p3 * (6300.0 / 1403.0)) * (sh / ch));
            b = (a * sh) / ch;
        }
    }
    const double xa[3] = {((460.0 * p2 + 451.0 * a) + 288.0 * b) / 1403.0,
                          ((460.0 * p2 - 891.0 * a) - 261.0 * b) / 1403.0,
                          ((460.0 * p2 - 220.0 * a) - 6300.0 * b) / 1403.0};
    Vec3 rc{};
    for (int i = 0; i < 3; ++i) {
        const double v = xa[i] - 0.1;
        const double av = std::fabs(v);
        const double beta = (27.13 * av) / (400.0 - av);
        const double pw = sgn(beta) * std::pow(std::fabs(beta), 1.0 / 0.42);
        rc[i] = (((100.0 / k.F_L) * sgn(v)) * pw) / k.D_rgb[i];
    }
    const Vec3 x100 = mat3_apply(k.m16_inv, rc);
    return {x100[0] / 100.0, x100[1] / 100.0, x100[2] / 100.0};
}

// C_max over 64 lightness rows (J' = 1 .. 110) and 720 hue columns: 18 bisection steps of the
// largest chroma whose inverse stays inside the output RGB cube (with 1e-6 slack).
std::vector<double> cam16_cmax_table(const Cam16Constants& k, const Mat3& m_to_rgb) {
    constexpr uint32_t kRows = 64, kCols = 720;
    std::vector<double> t(size_t(kRows) * kCols);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < int(kRows); ++i) {
        const double Jp = 1.0 + (109.0 * double(i)) / 63.0;
        for (uint32_t j = 0; j < kCols; ++j) {
            const double h = -M_PI + (2.0 * M_PI * double(j)) / 720.0;
            const double ch = std::cos(h), sh = std::sin(h);
            double lo = 0.0, hi = 150.0;
            for (int step = 0; step < 18; ++step) {
                const double mid = (lo + hi) / 2.0;
                const Vec3 xyz = cam16_inverse_unguarded(k, Jp, mid * ch, mid * sh);
                const Vec3 rgb = mat3_apply(m_to_rgb, xyz);
                bool in = true;
                for (double v : rgb) in = in && (v >= -1e-6 && v <= 1.0 + 1e-6);
                if (in) lo = mid;
                else hi = mid;
            }
            t[size_t(i) * kCols + j] = lo;
        }
    }
    return t;
}

std::shared_ptr<const Cam16Tables> Cam16Cache::get(const Resources& res, const std::string& space) {
    std::lock_guard<std::mutex> g(m_);
    auto it = by_space_.find(space);
    if (it != by_space_.end()) return it->second;
    if (!cctf_of(space)) fail_user("unknown colour space '" + space + "'");
    auto cs = colour_space(res.blob(), space);
    if (!cs) fail_user("colour space '" + space + "' has no baked matrices or whitepoint");
    if (cs->whitepoint[1] == 0.0) fail_user("colour space '" + space + "' has a whitepoint with y = 0");
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

// =============================== print set-up ====================================================

LiveParams LiveParams::from(const ParamSet& p) {
    LiveParams l;
    l.print_exposure = p.f(P::print_exposure);
    l.m_filter_shift = p.f(P::m_filter_shift);
    l.y_filter_shift = p.f(P::y_filter_shift);
    l.preflash_exposure = p.f(P::preflash_exposure);
    l.filter_shift_scale = p.f(P::filter_shift_scale);
    return l;
}

namespace {

// Fully inserted dichroic filters, k = 0 C, 1 M, 2 Y (reference src/print/setup.cpp:29-39).
std::array<Spectrum, 3> dichroic_filters() {
    std::array<Spectrum, 3> f{};
    for (size_t i = 0; i < 81; ++i) {
        const double l = 380.0 + 5.0 * double(i);
        f[2][i] = 0.5 * std::erf((l - 516.0) / 12.0) + 0.5;
        f[1][i] = l <= 550.0 ? 0.5 * (-std::erf((l - 500.0) / 8.0)) + 0.5 : 0.5 * std::erf((l - 610.0) / 8.0) + 0.5;
        f[0][i] = 0.5 * (-std::erf((l - 607.0) / 8.0)) + 0.5;
    }
    return f;
}

Spectrum filtered_light(const Spectrum& lamp, const std::array<Spectrum, 3>& filters, const Vec3& cc) {
    Vec3 tau{};
    for (int k = 0; k < 3; ++k) tau[k] = std::pow(10.0, -cc[k] / 100.0);
    Spectrum out{};
    for (size_t i = 0; i < 81; ++i) {
        double v = lamp[i];
        for (int k = 0; k < 3; ++k) v = v * (1.0 - (1.0 - filters[k][i]) * (1.0 - tau[k]));
        out[i] = v;
    }
    return out;
}

double exposure_factor(const Spectrum& density, const Spectrum& light, const std::array<double, 243>& sens) {
    Vec3 R{};
    for (size_t l = 0; l < 81; ++l) {
        double L = std::pow(10.0, -density[l]) * light[l];
        if (std::isnan(L)) L = 0.0;
        for (size_t c = 0; c < 3; ++c) R[c] += L * sens[3 * l + c];
    }
    double s = 0.0;
    for (size_t c = 0; c < 3; ++c) s += std::log(std::max(R[c], 1e-10));
    return 1.0 / std::exp((1.0 / 3.0) * s);
}

double mitchell64(double t) {
    constexpr double B = 1.0 / 3.0, C = 1.0 / 3.0;
    const double a = std::fabs(t);
    if (a < 1.0)
        return (1.0 / 6.0) * ((12.0 - 9.0 * B - 6.0 * C) * a * a * a + (-18.0 + 12.0 * B + 6.0 * C) * a * a + (6.0 - 2.0 * B));
    if (a < 2.0)
        return (1.0 / 6.0) * ((-B - 6.0 * C) * a * a * a + (6.0 * B + 30.0 * C) * a * a + (-12.0 * B - 48.0 * C) * a +
                              (8.0 * B + 24.0 * C));
    return 0.0;
}

struct Taps {
    int64_t idx[4];
    double w[4];
};

Taps mitchell_taps(double t, uint32_t L) {
    double u = t * double(L - 1);
    int64_t base;
    double frac;
    if (u <= 0.0) u = 0.0;
    if (u >= double(L - 1)) {
        base = int64_t(L) - 2;
        frac = 1.0;
    } else {
        base = int64_t(std::floor(u));
        frac = u - double(base);
    }
    Taps r{};
    for (int k = 0; k < 4; ++k) {
        int64_t n = base - 1 + k;
        if (n < 0) n = -n;
        if (n >= int64_t(L)) n = 2 * (int64_t(L) - 1) - n;
        r.idx[k] = n;
        r.w[k] = mitchell64(frac + 1.0 - double(k));
    }
    return r;
}

Spectrum probe_density(const Profile& film, const std::vector<double>& table, uint32_t L, const Mat3& srgb_to_xyz,
                       double gamma, double grey) {
    const Vec3 xyz = mat3_apply(srgb_to_xyz, {grey, grey, grey});
    const double b = (xyz[0] + xyz[1]) + xyz[2];
    const double bp = std::max(b, 1e-10);
    const double x = xyz[0] / bp, y = xyz[1] / bp;
    const double t0 = clip01((1.0 - x) * (1.0 - x));
    const double t1 = clip01(y / std::max(1.0 - x, 1e-10));
    const Vec3 s = bicubic_sample(table, L, t0, t1);
    const double bb = std::isnan(b) ? 0.0 : b;
    std::vector<double> axis(film.K());
    for (size_t k = 0; k < axis.size(); ++k) axis[k] = film.log_exposure[k] / gamma;
    Vec3 d{};
    for (size_t c = 0; c < 3; ++c) {
        const double raw = s[c] * bb;
        std::vector<double> curve(film.K());
        for (size_t i = 0; i < curve.size(); ++i) curve[i] = film.density_curves(i, c);
        d[c] = interp(std::log10(raw + 1e-10), axis, curve);
    }
    Spectrum D{};
    for (size_t l = 0; l < 81; ++l)
        D[l] = film.base_density[l] + ((d[0] * film.channel_density(l, 0) + d[1] * film.channel_density(l, 1)) +
                                       d[2] * film.channel_density(l, 2));
    return D;
}

void neutralise(std::array<double, 243>& eps, Spectrum& beta, std::array<double, 243>& wt) {
    for (size_t l = 0; l < 81; ++l) {
        bool bad = std::isnan(beta[l]);
        for (size_t c = 0; c < 3; ++c) bad = bad || std::isnan(eps[3 * l + c]) || std::isnan(wt[3 * l + c]);
        if (!bad) continue;
        beta[l] = 0.0;
        for (size_t c = 0; c < 3; ++c) eps[3 * l + c] = wt[3 * l + c] = 0.0;
    }
}

void narrow(float* dst, const double* src, size_t n) {
    for (size_t i = 0; i < n; ++i) dst[i] = f32(src[i]);
}

Spectrum need_illuminant(const Resources& res, const std::string& name, const char* what) {
    auto s = illuminant(res.blob(), name);
    if (!s) fail_user(std::string(what) + " '" + name + "' is not a known illuminant");
    return *s;
}

}  // namespace

Vec3 bicubic_sample(const std::vector<double>& table, uint32_t L, double t0, double t1) {
    const Taps a = mitchell_taps(t0, L), b = mitchell_taps(t1, L);
    Vec3 s{};
    double wsum = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            const double w = a.w[i] * b.w[j];
            const size_t base = (size_t(a.idx[i]) * L + size_t(b.idx[j])) * 3;
            for (int c = 0; c < 3; ++c) s[c] += w * table[base + c];
            wsum += w;
        }
    if (wsum != 0.0)
        for (double& v : s) v /= wsum;
    return s;
}

std::shared_ptr<PrintSetup> build_print_setup(const ParamSet& p, const FilmSetup& fs,
                                              std::shared_ptr<const Profile> paper_ptr, const Resources& res,
                                              Cam16Cache& cache, bool compensation) {
    const Profile& film = *fs.profile;
    const Profile& paper = *paper_ptr;
    const Blob& blob = res.blob();
    auto s = std::make_shared<PrintSetup>();
    s->params = p;
    s->paper = paper_ptr;
    s->scanned = p.b(P::scan_film);
    s->compensation = compensation;

    const std::string& out_name = p.s(P::output_color_space);
    if (!cctf_of(out_name)) fail_user("unknown colour space '" + out_name + "'");
    auto ocs = colour_space(blob, out_name);
    if (!ocs) fail_user("colour space '" + out_name + "' has no baked matrices");
    s->out_cs = *ocs;
    s->lamp = need_illuminant(res, p.s(P::enlarger_illuminant), "enlarger_illuminant");
    s->filters = dichroic_filters();
    s->neutral = {p.f(P::c_filter_neutral), p.f(P::m_filter_neutral), p.f(P::y_filter_neutral)};
    for (size_t l = 0; l < 81; ++l) {
        s->film_beta[l] = film.base_density[l];
        for (size_t c = 0; c < 3; ++c) s->film_eps[3 * l + c] = film.channel_density(l, c);
    }
    const std::vector<double> cmfs = blob.f64("colour/cmfs_1931_2deg");

    if (!s->scanned) {
        for (size_t l = 0; l < 81; ++l)
            for (size_t c = 0; c < 3; ++c) {
                const double v = std::pow(10.0, paper.log_sensitivity(l, c));
                s->paper_sens[3 * l + c] = std::isnan(v) ? 0.0 : v;
            }
        // the paper's characteristic curves from its cdfs model (reference src/print/setup.cpp:199-221)
        if (!paper.has_model || paper.model_type != "cdfs")
            fail_user("print profile '" + paper.id + "' has no density_curves_model of type cdfs");
        if (paper.amplitudes.rows < 3) fail_user("print profile '" + paper.id + "' has a malformed density_curves_model");
        const double sg = paper.positive() ? -1.0 : 1.0;
        const size_t K = paper.K();
        s->paper_K = uint32_t(K);
        s->paper_tab.assign(K * 5, 0.0f);
        for (size_t i = 0; i < K; ++i) {
            const double x = paper.log_exposure[i];
            s->paper_tab[i] = f32(x);
            if (i + 1 < K) {
                const double d = paper.log_exposure[i + 1] - paper.log_exposure[i];
                s->paper_tab[K + i] = d == 0.0 ? 0.0f : f32(1.0 / d);
            }
            for (size_t c = 0; c < 3; ++c) {
                double v = 0.0;
                for (size_t l = 0; l < paper.amplitudes.cols; ++l) {
                    const double z = (sg * (x - paper.centers(c, l))) / paper.sigmas(c, l);
                    v += paper.amplitudes(c, l) * (0.5 * std::erfc(-z / std::sqrt(2.0)));
                }
                s->paper_tab[2 * K + 3 * i + c] = f32(v);
                s->paper_y64.push_back(v);
            }
        }
        auto srgb = colour_space(blob, "sRGB");
        auto cat16 = cat_matrix(blob, "CAT16");
        if (!srgb || !cat16) fail_user("the constants blob lacks sRGB or CAT16 (needed by the mid-grey probe)");
        const Spectrum ref = need_illuminant(res, film.reference_illuminant, "the film's reference_illuminant");
        Mat3 pm = srgb->rgb_to_xyz;
        if (auto a = von_kries(srgb->whitepoint, chromaticity(blob, ref), *cat16, Guard::Source))
            pm = mat3_mul(*a, srgb->rgb_to_xyz);
        const double gamma = p.f(P::density_curve_gamma);
        s->probe_mid = probe_density(film, fs.table64, fs.L, pm, gamma, 0.184);
        if (compensation)
            s->probe_comp = probe_density(film, fs.table64, fs.L, pm, gamma, 0.184 * std::exp2(p.f(P::exposure_compensation_ev)));
    }

    const Profile& medium = s->scanned ? film : paper;
    const Spectrum view = need_illuminant(res, medium.viewing_illuminant, "viewing_illuminant");
    {
        double N = 0.0;
        for (size_t l = 0; l < 81; ++l) N += view[l] * cmfs[3 * l + 1];
        Vec3 sum{};
        for (size_t l = 0; l < 81; ++l)
            for (size_t k = 0; k < 3; ++k) {
                s->scan_wt[3 * l + k] = (view[l] * cmfs[3 * l + k]) / N;
                sum[k] += view[l] * cmfs[3 * l + k];
            }
        for (size_t k = 0; k < 3; ++k) s->view_xyz[k] = sum[k] / N;
        for (size_t l = 0; l < 81; ++l) {
            s->scan_beta[l] = medium.base_density[l];
            for (size_t c = 0; c < 3; ++c) s->scan_eps[3 * l + c] = medium.channel_density(l, c);
        }
        neutralise(s->scan_eps, s->scan_beta, s->scan_wt);
        narrow(s->scan32.eps, s->scan_eps.data(), 243);
        narrow(s->scan32.beta, s->scan_beta.data(), 81);
        narrow(s->scan32.wt, s->scan_wt.data(), 243);
    }
    s->scanner_lens_blur_px = p.f(P::scanner_lens_blur);
    s->levels_black = p.b(P::scanner_black_correction);
    s->levels_white = p.b(P::scanner_white_correction);
    s->levels_B = 0.01 / 12.92;
    s->levels_W = std::pow((0.98 + 0.055) / 1.055, 2.4);
    s->film_positive = film.positive();
    s->paper_positive = paper.positive();
    for (size_t c = 0; c < 3; ++c) {  // the film's white density: the density curve's largest value (NaN skipped)
        double m = std::numeric_limits<double>::quiet_NaN();
        for (size_t k = 0; k < film.density_curves.rows; ++k) {
            const double v = film.density_curves(k, c);
            if (!std::isnan(v) && (std::isnan(m) || v > m)) m = v;
        }
        s->film_white_density[c] = m;
    }
    if (!s->scanned) {  // the paper's mean curve and mean base (NaN skipped)
        auto nanmean = [](const double* v, size_t n, size_t stride) {
            double sum = 0.0;
            size_t k = 0;
            for (size_t i = 0; i < n; ++i)
                if (!std::isnan(v[i * stride])) {
                    sum += v[i * stride];
                    ++k;
                }
            return k ? sum / double(k) : std::numeric_limits<double>::quiet_NaN();
        };
        s->paper_mean_curve.resize(paper.K());
        for (size_t i = 0; i < paper.K(); ++i) s->paper_mean_curve[i] = nanmean(&paper.density_curves.v[3 * i], 3, 1);
        s->paper_mean_base = nanmean(paper.base_density.data(), paper.base_density.size(), 1);
    }
    s->edr = p.b(P::extended_dynamic_range);
    if (s->edr) {
        if (!paper.edr) fail_user("extended_dynamic_range: print profile '" + paper.id + "' has no valid edr_tone_map");
        s->edr_lo = paper.edr->lo;
        s->edr_hi = paper.edr->hi;
        s->edr_toe = paper.edr->toe;
        s->edr_shoulder = paper.edr->shoulder;
        s->edr_tab.resize(paper.edr->target.size());
        for (size_t i = 0; i < s->edr_tab.size(); ++i) s->edr_tab[i] = f32(paper.edr->target[i]);
    }
    s->glare = p.b(P::glare_active);
    s->glare_amount = p.f(P::glare_amount);
    s->glare_tint = s->view_xyz;  // a printed frame's viewing illuminant (the only case that adds glare)
    {
        auto cat02 = cat_matrix(blob, "CAT02");
        if (!cat02) fail_user("the constants blob lacks colour/cat/CAT02");
        const Vec3& w = s->view_xyz;
        const double sum = (w[0] + w[1]) + w[2];
        const std::array<double, 2> xy_view = {w[0] / sum, w[1] / sum};
        Mat3 m = s->out_cs.xyz_to_rgb;
        if (auto a = von_kries(xy_view, s->out_cs.whitepoint, *cat02, Guard::Target)) m = mat3_mul(m, *a);
        narrow(s->to_rgb, m.data(), 9);
        s->to_rgb64 = m;
    }
    s->cam = cache.get(res, out_name);
    {
        const Cam16Tables& t = *s->cam;
        const Cam16Constants& c = t.k;
        Cam16Args& q = s->cam_args;
        q.rows = 64;
        q.cols = 720;
        narrow(q.m_to_xyz, t.m_to_xyz.data(), 9);
        narrow(q.m_to_rgb, t.m_to_rgb.data(), 9);
        narrow(q.m16, kM16.data(), 9);
        narrow(q.m16_inv, kM16InvPublished.data(), 9);
        for (int i = 0; i < 3; ++i) q.d_rgb[i] = f32(c.D_rgb[i]);
        q.f_l = f32(c.F_L);
        q.n_bb = f32(c.N_bb);
        q.n_cb = f32(c.N_cb);
        q.n = f32(c.n);
        q.z = f32(c.z);
        q.a_w = f32(c.A_w);
        q.c = f32(c.c);
        q.n_c = f32(c.N_c);
        q.j_first = f32(1.0);
        q.j_last = f32(110.0);
        q.h_first = f32(-M_PI);
        q.h_step = f32(2.0 * M_PI / 720.0);
        const double knee[3] = {0, 1, 6}, lc[3] = {0.7, 1.0, 2.2};
        for (int i = 0; i < 3; ++i) {
            q.knee[i] = f32(knee[i]);
            q.lc[i] = f32(lc[i]);
        }
        q.lc_active = 1;
        q.j_white = f32(c.J_white);
        // the kernel's per-pixel constants in binary32, the operations of print.metal:53-64
        q.cz = q.c * q.z;
        q.inv_cz = 1.0f / q.cz;
        q.f_l_qrt = std::pow(q.f_l, 0.25f);
        q.chroma_k = std::pow(1.64f - std::pow(0.29f, q.n), 0.73f);
        q.hundred_over_f_l = 100.0f / q.f_l;
        q.inv_a_w = 1.0f / q.a_w;
        q.inv_j_white = 1.0f / q.j_white;
        q.inv_n_bb = 1.0f / q.n_bb;
        q.inv_f_l_qrt = 1.0f / q.f_l_qrt;
        q.inv_h_step = 1.0f / q.h_step;
        q.inv_j_span = 1.0f / (q.j_last - q.j_first);
        for (int i = 0; i < 3; ++i) q.inv_d_rgb[i] = 1.0f / q.d_rgb[i];
        q.knee_inv_span = 1.0f / (q.knee[1] - q.knee[0]);
        q.knee_inv_p = 1.0f / q.knee[2];
        q.lc_inv_span = 1.0f / (q.lc[1] - q.lc[0]);
        q.lc_inv_p = 1.0f / q.lc[2];
    }
    s->cctf = p.b(P::output_cctf_encoding);
    s->cctf_mode = uint32_t(s->out_cs.cctf);
    {
        const Mat3 nid = mat3_mul(s->out_cs.xyz_to_rgb, s->out_cs.rgb_to_xyz);
        narrow(s->m_nid, nid.data(), 9);
        s->m_nid64 = nid;
    }
    return s;
}

namespace {
// The Y that a film density triple d prints to (reference src/print/setup.cpp:281-314): the enlarger
// integral, the paper's log exposure, its density curves, then the scan integral's Y with the narrowed
// scan tables; max(y, 0) + 1e-10.
double reference_y(const PrintSetup& s, const PrintRun& r, const Vec3& d) {
    constexpr double kLog2Of10 = 3.32192809488736234787;
    const Profile& paper = *s.paper;
    Vec3 ell{};
    {
        Vec3 R{};
        for (size_t l = 0; l < 81; ++l) {
            const double D = r.beta_n[l] + ((d[0] * r.eps_n[3 * l] + d[1] * r.eps_n[3 * l + 1]) + d[2] * r.eps_n[3 * l + 2]);
            const double T = std::exp2(-D * kLog2Of10);
            for (size_t c = 0; c < 3; ++c) R[c] += T * r.w_n[3 * l + c];
        }
        for (size_t c = 0; c < 3; ++c) ell[c] = std::log10(std::max(R[c] * r.g[c] + r.o[c], 0.0) + 1e-10);
    }
    Vec3 Dp{};
    for (size_t c = 0; c < 3; ++c) {
        std::vector<double> curve(paper.density_curves.rows);
        for (size_t i = 0; i < curve.size(); ++i) curve[i] = paper.density_curves(i, c);
        Dp[c] = interp(ell[c], paper.log_exposure, curve);
    }
    const SpectralTables& a = s.scan32;
    double y = 0.0;
    for (size_t l = 0; l < 81; ++l) {
        const double D = ((Dp[0] * double(a.eps[3 * l]) + Dp[1] * double(a.eps[3 * l + 1])) + Dp[2] * double(a.eps[3 * l + 2])) +
                         double(a.beta[l]);
        y += std::exp2(-D * kLog2Of10) * double(a.wt[3 * l + 1]);
    }
    return std::max(y, 0.0) + 1e-10;
}
}  // namespace

PrintRun compute_run(const PrintSetup& s, const LiveParams& live) {
    PrintRun r;
    if (!s.scanned) {
        const Vec3 cc = {s.neutral[0], s.neutral[1] + live.m_filter_shift * live.filter_shift_scale,
                         s.neutral[2] + live.y_filter_shift * live.filter_shift_scale};
        r.light = filtered_light(s.lamp, s.filters, cc);
        r.eps_n = s.film_eps;
        r.beta_n = s.film_beta;
        for (size_t l = 0; l < 81; ++l)
            for (size_t c = 0; c < 3; ++c) r.w_n[3 * l + c] = r.light[l] * s.paper_sens[3 * l + c];
        neutralise(r.eps_n, r.beta_n, r.w_n);
        const double phi = s.compensation ? exposure_factor(s.probe_comp, r.light, s.paper_sens)
                                          : exposure_factor(s.probe_mid, r.light, s.paper_sens);
        r.g = {phi, phi, phi};
        if (live.preflash_exposure > 0.0) {
            const Spectrum pre = filtered_light(s.lamp, s.filters, s.neutral);
            Vec3 sum{};
            for (size_t l = 0; l < 81; ++l) {
                double L = std::pow(10.0, -s.film_beta[l]) * pre[l];
                if (std::isnan(L)) L = 0.0;
                for (size_t c = 0; c < 3; ++c) sum[c] += L * s.paper_sens[3 * l + c];
            }
            for (size_t c = 0; c < 3; ++c) r.o[c] = live.preflash_exposure * sum[c];
        }
    }
    // scanner levels (reference src/print/setup.cpp:371-390): the print's Y of the film's black and
    // white densities, the line through the targets, and the exposure correction that keeps mid grey
    r.levels = s.levels_active();
    if (r.levels) {
        if (!s.scanned && !s.paper_positive) {
            r.y_k = reference_y(s, r, {-0.03, -0.03, -0.03});
            r.y_w = reference_y(s, r, s.film_white_density);
        }
        double B = s.levels_B, W = s.levels_W;
        if (s.levels_black && !s.levels_white) W = r.y_w;
        if (s.levels_white && !s.levels_black) B = r.y_k;
        r.m = (W - B) / (r.y_w - r.y_k + 1e-10);
        r.q = B - r.m * r.y_k;
        if (!s.scanned && !s.paper_positive) {
            const Profile& paper = *s.paper;
            const double mid = 0.184;
            const double g_star = (mid - r.q) / r.m;
            const double e_star = interp(-std::log10(g_star) - s.paper_mean_base, s.paper_mean_curve, paper.log_exposure);
            const double e_0 = interp(-std::log10(mid) - s.paper_mean_base, s.paper_mean_curve, paper.log_exposure);
            r.kappa_bw = std::pow(10.0, e_star - e_0);
        }
    }
    r.k_gain = f32(live.print_exposure * r.kappa_bw);
    narrow(r.enl32.eps, r.eps_n.data(), 243);
    narrow(r.enl32.beta, r.beta_n.data(), 81);
    narrow(r.enl32.wt, r.w_n.data(), 243);
    return r;
}

}  // namespace spkb
