// The print side's binary64 set-up (reference src/print/build.cpp:53-236, src/print/setup.cpp:29-399):
// per pipeline, what the enlarger, the paper, the scanner and the output need (build_print_setup); per print,
// the enlarger light for the live filter settings and the exposure that keeps mid grey (compute_run).
//
// Model pieces, each a function below:
//   * the enlarger: a lamp through three dichroic filters (erf band edges), each inserted by its CC value;
//   * the exposure factor: the reciprocal geometric mean over the paper layers of the exposure a probe
//     density receives, the probe being the film's density for a mid-grey (18.4 %) sRGB patch;
//   * the paper: characteristic curves from its model of normal-CDF components;
//   * the scan: the viewing illuminant's CIE 1931 weights normalised to Y = 1;
//   * scanner levels: black and white targets through the print's own Y of the film's extreme densities;
//   * the output: XYZ -> output RGB with the CAT02 adaptation from the viewing white, and the binary32
//     constants of the CAM16-UCS gamut compression.
// The floating-point expressions keep the reference's operation order, so the narrowed tables are the
// reference's bit for bit; the decomposition, names and messages are this file's.
#include <cmath>
#include <limits>

#include "setup.hpp"
#include "status.hpp"

namespace spkb {

namespace {

constexpr size_t kBins = 81;
constexpr double kMidGrey = 0.184;
constexpr double kLog2Of10 = 3.32192809488736234787;

double bin_nm(size_t b) { return 380.0 + 5.0 * double(b); }

// ---- the enlarger ----

// one erf band edge, 0 -> 1 across `centre` (rising) or 1 -> 0 (falling), of the given width
double band_edge(double nm, double centre, double width, bool rising) {
    const double e = std::erf((nm - centre) / width);
    return rising ? 0.5 * e + 0.5 : 0.5 * (-e) + 0.5;
}

// the fully inserted transmittance of the cyan (0), magenta (1) and yellow (2) filters
std::array<Spectrum, 3> dichroic_set() {
    std::array<Spectrum, 3> f{};
    for (size_t b = 0; b < kBins; ++b) {
        const double nm = bin_nm(b);
        f[0][b] = band_edge(nm, 607.0, 8.0, false);                                             // passes blue-green
        f[1][b] = nm <= 550.0 ? band_edge(nm, 500.0, 8.0, false) : band_edge(nm, 610.0, 8.0, true);  // a green notch
        f[2][b] = band_edge(nm, 516.0, 12.0, true);                                             // passes green-red
    }
    return f;
}

// the lamp through the filters at CC values cc (a filter at CC v passes 10^(-v/100) of the band it blocks)
Spectrum enlarger_light(const Spectrum& lamp, const std::array<Spectrum, 3>& filters, const Vec3& cc) {
    Vec3 pass{};
    for (size_t k = 0; k < 3; ++k) pass[k] = std::pow(10.0, -cc[k] / 100.0);
    Spectrum out{};
    for (size_t b = 0; b < kBins; ++b) {
        double v = lamp[b];
        for (size_t k = 0; k < 3; ++k) v = v * (1.0 - (1.0 - filters[k][b]) * (1.0 - pass[k]));
        out[b] = v;
    }
    return out;
}

// the exposure each paper layer receives through film density D(l): sum_l 10^-D(l) light(l) sens_c(l)
Vec3 layer_exposure(const Spectrum& density, const Spectrum& light, const std::array<double, 243>& sens) {
    Vec3 e{};
    for (size_t b = 0; b < kBins; ++b) {
        double through = std::pow(10.0, -density[b]) * light[b];
        if (std::isnan(through)) through = 0.0;
        for (size_t c = 0; c < 3; ++c) e[c] += through * sens[3 * b + c];
    }
    return e;
}

// 1 / (the geometric mean of the three layer exposures of the probe density)
double exposure_factor(const Spectrum& probe, const Spectrum& light, const std::array<double, 243>& sens) {
    const Vec3 e = layer_exposure(probe, light, sens);
    double log_sum = 0.0;
    for (size_t c = 0; c < 3; ++c) log_sum += std::log(std::max(e[c], 1e-10));
    return 1.0 / std::exp((1.0 / 3.0) * log_sum);
}

// ---- the mid-grey probe ----

// the Mitchell-Netravali cubic, B = C = 1/3
double mitchell_weight(double t) {
    constexpr double B = 1.0 / 3.0, C = 1.0 / 3.0;
    const double a = std::fabs(t);
    if (a < 1.0)
        return (1.0 / 6.0) * ((12.0 - 9.0 * B - 6.0 * C) * a * a * a + (-18.0 + 12.0 * B + 6.0 * C) * a * a + (6.0 - 2.0 * B));
    if (a < 2.0)
        return (1.0 / 6.0) * ((-B - 6.0 * C) * a * a * a + (6.0 * B + 30.0 * C) * a * a + (-12.0 * B - 48.0 * C) * a +
                              (8.0 * B + 24.0 * C));
    return 0.0;
}

// the four taps of one axis at coordinate t in [0, 1]: indices reflected at the ends, and weights
struct AxisTaps {
    int64_t idx[4];
    double w[4];
};
AxisTaps axis_taps(double t, uint32_t L) {
    const double last = double(L - 1);
    double u = t * last;
    if (u <= 0.0) u = 0.0;
    int64_t base = int64_t(L) - 2;
    double frac = 1.0;
    if (u < last) {
        base = int64_t(std::floor(u));
        frac = u - double(base);
    }
    AxisTaps a{};
    for (int k = 0; k < 4; ++k) {
        int64_t i = base - 1 + k;
        if (i < 0) i = -i;
        if (i >= int64_t(L)) i = 2 * (int64_t(L) - 1) - i;
        a.idx[k] = i;
        a.w[k] = mitchell_weight(frac + 1.0 - double(k));
    }
    return a;
}

// the film's spectral density for a grey sRGB patch of linear value `grey`: its XYZ (probe_matrix: sRGB ->
// XYZ under the film's reference illuminant), the upsampling table at its chromaticity, the layer curves
Spectrum grey_patch_density(const Profile& film, const std::vector<double>& table, uint32_t L, const Mat3& probe_matrix,
                            double gamma, double grey) {
    const Vec3 xyz = mat3_apply(probe_matrix, {grey, grey, grey});
    const double sum = (xyz[0] + xyz[1]) + xyz[2];
    const double div = std::max(sum, 1e-10);
    const double x = xyz[0] / div, y = xyz[1] / div;
    const double o = 1.0 - x;
    const double t0 = std::min(std::max(o * o, 0.0), 1.0);
    const double t1 = std::min(std::max(y / std::max(o, 1e-10), 0.0), 1.0);
    const Vec3 response = bicubic_sample(table, L, t0, t1);
    const double scale = std::isnan(sum) ? 0.0 : sum;
    std::vector<double> log_h(film.K());
    for (size_t k = 0; k < log_h.size(); ++k) log_h[k] = film.log_exposure[k] / gamma;
    Vec3 layer{};
    for (size_t c = 0; c < 3; ++c) {
        std::vector<double> curve(film.K());
        for (size_t i = 0; i < curve.size(); ++i) curve[i] = film.density_curves(i, c);
        layer[c] = interp(std::log10(response[c] * scale + 1e-10), log_h, curve);
    }
    Spectrum D{};
    for (size_t b = 0; b < kBins; ++b)
        D[b] = film.base_density[b] + ((layer[0] * film.channel_density(b, 0) + layer[1] * film.channel_density(b, 1)) +
                                       layer[2] * film.channel_density(b, 2));
    return D;
}

// a bin whose base, layer density or weight is undefined contributes nothing
void drop_undefined_bins(std::array<double, 243>& eps, Spectrum& beta, std::array<double, 243>& wt) {
    for (size_t b = 0; b < kBins; ++b) {
        bool undefined = std::isnan(beta[b]);
        for (size_t c = 0; c < 3; ++c) undefined = undefined || std::isnan(eps[3 * b + c]) || std::isnan(wt[3 * b + c]);
        if (!undefined) continue;
        beta[b] = 0.0;
        for (size_t c = 0; c < 3; ++c) eps[3 * b + c] = wt[3 * b + c] = 0.0;
    }
}

template <size_t N>
void to_f32(float* dst, const std::array<double, N>& src) {
    for (size_t i = 0; i < N; ++i) dst[i] = f32(src[i]);
}

Spectrum named_illuminant(const Resources& res, const std::string& name, const char* role) {
    const std::optional<Spectrum> s = illuminant(res.blob(), name);
    if (!s) fail_user(std::string(role) + ": no illuminant called '" + name + "' in the resources");
    return *s;
}

double nan_skipping_mean(const double* v, size_t n, size_t stride) {
    double sum = 0.0;
    size_t k = 0;
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(v[i * stride])) {
            sum += v[i * stride];
            ++k;
        }
    return k ? sum / double(k) : std::numeric_limits<double>::quiet_NaN();
}

// ---- pieces of build_print_setup ----

// the paper's characteristic curves from its model: d_c(x) = sum_l a_cl Phi(s (x - mu_cl) / sigma_cl), with
// s = -1 for a positive paper; tabulated on its log-exposure axis as x[K] | 1 / dx[K] | y[K][3]
void paper_curves(const Profile& paper, PrintSetup& s) {
    if (!paper.has_model || paper.model_type != "cdfs")
        fail_user("print stock '" + paper.id + "': the print needs a density_curves_model made of normal CDFs (cdfs)");
    if (paper.amplitudes.rows < 3)
        fail_user("print stock '" + paper.id + "': its density_curves_model needs a row per colour channel");
    const double dir = paper.positive() ? -1.0 : 1.0;
    const size_t K = paper.K();
    s.paper_K = uint32_t(K);
    s.paper_tab.assign(K * 5, 0.0f);
    for (size_t i = 0; i < K; ++i) {
        const double x = paper.log_exposure[i];
        s.paper_tab[i] = f32(x);
        if (i + 1 < K) {
            const double dx = paper.log_exposure[i + 1] - paper.log_exposure[i];
            s.paper_tab[K + i] = dx == 0.0 ? 0.0f : f32(1.0 / dx);
        }
        for (size_t c = 0; c < 3; ++c) {
            double d = 0.0;
            for (size_t l = 0; l < paper.amplitudes.cols; ++l) {
                const double z = (dir * (x - paper.centers(c, l))) / paper.sigmas(c, l);
                d += paper.amplitudes(c, l) * (0.5 * std::erfc(-z / std::sqrt(2.0)));
            }
            s.paper_tab[2 * K + 3 * i + c] = f32(d);
            s.paper_y64.push_back(d);
        }
    }
}

// the scan integral's tables: the viewed medium's densities and the viewing illuminant's CIE 1931 weights,
// normalised so that the illuminant itself has Y = 1 (view_xyz: its XYZ at that scale)
void scan_tables(const Profile& medium, const Spectrum& view, const std::vector<double>& cmf, PrintSetup& s) {
    double norm = 0.0;
    for (size_t b = 0; b < kBins; ++b) norm += view[b] * cmf[3 * b + 1];
    Vec3 total{};
    for (size_t b = 0; b < kBins; ++b)
        for (size_t k = 0; k < 3; ++k) {
            s.scan_wt[3 * b + k] = (view[b] * cmf[3 * b + k]) / norm;
            total[k] += view[b] * cmf[3 * b + k];
        }
    for (size_t k = 0; k < 3; ++k) s.view_xyz[k] = total[k] / norm;
    for (size_t b = 0; b < kBins; ++b) {
        s.scan_beta[b] = medium.base_density[b];
        for (size_t c = 0; c < 3; ++c) s.scan_eps[3 * b + c] = medium.channel_density(b, c);
    }
    drop_undefined_bins(s.scan_eps, s.scan_beta, s.scan_wt);
    to_f32(s.scan32.eps, s.scan_eps);
    to_f32(s.scan32.beta, s.scan_beta);
    to_f32(s.scan32.wt, s.scan_wt);
}

// the constants scanner levels need at print time
void levels_targets(const Profile& film, const Profile& paper, const ParamSet& p, PrintSetup& s) {
    s.levels_black = p.b(P::scanner_black_correction);
    s.levels_white = p.b(P::scanner_white_correction);
    s.levels_B = 0.01 / 12.92;                              // the sRGB code value 0.01, linear
    s.levels_W = std::pow((0.98 + 0.055) / 1.055, 2.4);     // the sRGB code value 0.98, linear
    s.film_positive = film.positive();
    s.paper_positive = paper.positive();
    for (size_t c = 0; c < 3; ++c) {  // the film's white: the largest value of its density curve
        double top = std::numeric_limits<double>::quiet_NaN();
        for (size_t k = 0; k < film.density_curves.rows; ++k) {
            const double v = film.density_curves(k, c);
            if (!std::isnan(v) && (std::isnan(top) || v > top)) top = v;
        }
        s.film_white_density[c] = top;
    }
    if (s.scanned) return;
    s.paper_mean_curve.resize(paper.K());
    for (size_t i = 0; i < paper.K(); ++i) s.paper_mean_curve[i] = nan_skipping_mean(&paper.density_curves.v[3 * i], 3, 1);
    s.paper_mean_base = nan_skipping_mean(paper.base_density.data(), paper.base_density.size(), 1);
}

// XYZ (viewing white) -> output RGB, with CAT02 from the viewing white to the output space's white
Mat3 output_matrix(const Blob& blob, const ColourSpace& out, const Vec3& view_xyz) {
    const std::optional<Mat3> cat02 = cat_matrix(blob, "CAT02");
    if (!cat02) fail_user("output transform: the resources have no colour/cat/CAT02 matrix");
    const double sum = (view_xyz[0] + view_xyz[1]) + view_xyz[2];
    const std::array<double, 2> view_white = {view_xyz[0] / sum, view_xyz[1] / sum};
    Mat3 m = out.xyz_to_rgb;
    if (const std::optional<Mat3> a = von_kries(view_white, out.whitepoint, *cat02, Guard::Target)) m = mat3_mul(m, *a);
    return m;
}

// the gamut compression's kernel arguments: the model's constants in binary32 and the per-pixel constants
// the kernel derives from them, formed here in binary32 with the same operations
Cam16Args gamut_args(const Cam16Tables& t, const Mat3& m16, const Mat3& m16_inv_published) {
    const Cam16Constants& k = t.k;
    Cam16Args q{};
    q.rows = 64;
    q.cols = 720;
    to_f32(q.m_to_xyz, t.m_to_xyz);
    to_f32(q.m_to_rgb, t.m_to_rgb);
    to_f32(q.m16, m16);
    to_f32(q.m16_inv, m16_inv_published);
    for (int i = 0; i < 3; ++i) q.d_rgb[i] = f32(k.D_rgb[i]);
    q.f_l = f32(k.F_L);
    q.n_bb = f32(k.N_bb);
    q.n_cb = f32(k.N_cb);
    q.n = f32(k.n);
    q.z = f32(k.z);
    q.a_w = f32(k.A_w);
    q.c = f32(k.c);
    q.n_c = f32(k.N_c);
    q.j_first = f32(1.0);
    q.j_last = f32(110.0);
    q.h_first = f32(-M_PI);
    q.h_step = f32(2.0 * M_PI / 720.0);
    constexpr double chroma_knee[3] = {0.0, 1.0, 6.0}, lightness_knee[3] = {0.7, 1.0, 2.2};  // threshold, limit, power
    for (int i = 0; i < 3; ++i) {
        q.knee[i] = f32(chroma_knee[i]);
        q.lc[i] = f32(lightness_knee[i]);
    }
    q.lc_active = 1;
    q.j_white = f32(k.J_white);
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
    return q;
}

}  // namespace

LiveParams LiveParams::from(const ParamSet& p) {
    LiveParams l;
    l.print_exposure = p.f(P::print_exposure);
    l.m_filter_shift = p.f(P::m_filter_shift);
    l.y_filter_shift = p.f(P::y_filter_shift);
    l.preflash_exposure = p.f(P::preflash_exposure);
    l.filter_shift_scale = p.f(P::filter_shift_scale);
    return l;
}

Vec3 bicubic_sample(const std::vector<double>& table, uint32_t L, double t0, double t1) {
    const AxisTaps a = axis_taps(t0, L), b = axis_taps(t1, L);
    Vec3 acc{};
    double wsum = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            const double w = a.w[i] * b.w[j];
            const double* texel = &table[(size_t(a.idx[i]) * L + size_t(b.idx[j])) * 3];
            for (int c = 0; c < 3; ++c) acc[c] += w * texel[c];
            wsum += w;
        }
    if (wsum != 0.0)
        for (double& v : acc) v /= wsum;
    return acc;
}

std::shared_ptr<PrintSetup> build_print_setup(const ParamSet& p, const FilmSetup& fs,
                                              std::shared_ptr<const Profile> paper_ptr, const Resources& res,
                                              Cam16Cache& cache, bool compensation) {
    static constexpr Mat3 kCat16Cone = {0.401288, 0.650173,  -0.051461, -0.250268, 1.204414,
                                        0.045854, -0.002079, 0.048952,  0.953127};
    static constexpr Mat3 kCat16ConeInverse8 = {1.86206786,  -1.01125463, 0.14918677,  0.38752654, 0.62144744,
                                                -0.00897398, -0.01584150, -0.03412294, 1.04996444};
    const Profile& film = *fs.profile;
    const Profile& paper = *paper_ptr;
    const Blob& blob = res.blob();
    auto s = std::make_shared<PrintSetup>();
    s->params = p;
    s->paper = paper_ptr;
    s->scanned = p.b(P::scan_film);
    s->compensation = compensation;

    const std::string& out_name = p.s(P::output_color_space);
    if (!cctf_of(out_name)) fail_user("output_color_space: '" + out_name + "' is not one of the known colour spaces");
    const std::optional<ColourSpace> out = colour_space(blob, out_name);
    if (!out) fail_user("output_color_space: the resources have no matrices for '" + out_name + "'");
    s->out_cs = *out;

    // the enlarger and the film it prints through
    s->lamp = named_illuminant(res, p.s(P::enlarger_illuminant), "enlarger_illuminant");
    s->filters = dichroic_set();
    s->neutral = {p.f(P::c_filter_neutral), p.f(P::m_filter_neutral), p.f(P::y_filter_neutral)};
    for (size_t b = 0; b < kBins; ++b) {
        s->film_beta[b] = film.base_density[b];
        for (size_t c = 0; c < 3; ++c) s->film_eps[3 * b + c] = film.channel_density(b, c);
    }
    const std::vector<double> cmf = blob.f64("colour/cmfs_1931_2deg");

    if (!s->scanned) {
        for (size_t b = 0; b < kBins; ++b)
            for (size_t c = 0; c < 3; ++c) {
                const double v = std::pow(10.0, paper.log_sensitivity(b, c));
                s->paper_sens[3 * b + c] = std::isnan(v) ? 0.0 : v;
            }
        paper_curves(paper, *s);
        // the mid-grey probe: sRGB under the film's reference illuminant (CAT16 from sRGB's white)
        const std::optional<ColourSpace> srgb = colour_space(blob, "sRGB");
        const std::optional<Mat3> cat16 = cat_matrix(blob, "CAT16");
        if (!srgb || !cat16) fail_user("exposure factor: the mid-grey probe needs the sRGB space and CAT16 in the resources");
        const Spectrum ref_light = named_illuminant(res, film.reference_illuminant, "film reference_illuminant");
        Mat3 probe_matrix = srgb->rgb_to_xyz;
        if (const std::optional<Mat3> a = von_kries(srgb->whitepoint, chromaticity(blob, ref_light), *cat16, Guard::Source))
            probe_matrix = mat3_mul(*a, srgb->rgb_to_xyz);
        const double gamma = p.f(P::density_curve_gamma);
        s->probe_mid = grey_patch_density(film, fs.table64, fs.L, probe_matrix, gamma, kMidGrey);
        if (compensation)
            s->probe_comp = grey_patch_density(film, fs.table64, fs.L, probe_matrix, gamma,
                                               kMidGrey * std::exp2(p.f(P::exposure_compensation_ev)));
    }

    const Profile& medium = s->scanned ? film : paper;
    scan_tables(medium, named_illuminant(res, medium.viewing_illuminant, "viewing_illuminant"), cmf, *s);
    s->scanner_lens_blur_px = p.f(P::scanner_lens_blur);
    levels_targets(film, paper, p, *s);
    s->edr = p.b(P::extended_dynamic_range);
    if (s->edr) {
        if (!paper.edr)
            fail_user("extended_dynamic_range: print stock '" + paper.id + "' carries no usable edr_tone_map");
        s->edr_lo = paper.edr->lo;
        s->edr_hi = paper.edr->hi;
        s->edr_toe = paper.edr->toe;
        s->edr_shoulder = paper.edr->shoulder;
        s->edr_tab.resize(paper.edr->target.size());
        for (size_t i = 0; i < s->edr_tab.size(); ++i) s->edr_tab[i] = f32(paper.edr->target[i]);
    }
    s->glare = p.b(P::glare_active);
    s->glare_amount = p.f(P::glare_amount);
    s->glare_tint = s->view_xyz;  // glare is added to printed frames only, seen under the viewing illuminant
    s->to_rgb64 = output_matrix(blob, s->out_cs, s->view_xyz);
    to_f32(s->to_rgb, s->to_rgb64);
    s->cam = cache.get(res, out_name);
    s->cam_args = gamut_args(*s->cam, kCat16Cone, kCat16ConeInverse8);
    s->cctf = p.b(P::output_cctf_encoding);
    s->cctf_mode = uint32_t(s->out_cs.cctf);
    s->m_nid64 = mat3_mul(s->out_cs.xyz_to_rgb, s->out_cs.rgb_to_xyz);
    to_f32(s->m_nid, s->m_nid64);
    return s;
}

namespace {

// The Y that film densities d print to (reference src/print/setup.cpp:281-314): the enlarger integral and
// the paper's log exposure in binary64, its density curves, then the scan integral's Y from the narrowed
// scan tables; max(Y, 0) + 1e-10.
double printed_y(const PrintSetup& s, const PrintRun& r, const Vec3& d) {
    const Profile& paper = *s.paper;
    Vec3 log_e{};
    {
        Vec3 R{};
        for (size_t b = 0; b < kBins; ++b) {
            const double D = r.beta_n[b] + ((d[0] * r.eps_n[3 * b] + d[1] * r.eps_n[3 * b + 1]) + d[2] * r.eps_n[3 * b + 2]);
            const double T = std::exp2(-D * kLog2Of10);
            for (size_t c = 0; c < 3; ++c) R[c] += T * r.w_n[3 * b + c];
        }
        for (size_t c = 0; c < 3; ++c) log_e[c] = std::log10(std::max(R[c] * r.g[c] + r.o[c], 0.0) + 1e-10);
    }
    Vec3 paper_d{};
    for (size_t c = 0; c < 3; ++c) {
        std::vector<double> curve(paper.density_curves.rows);
        for (size_t i = 0; i < curve.size(); ++i) curve[i] = paper.density_curves(i, c);
        paper_d[c] = interp(log_e[c], paper.log_exposure, curve);
    }
    const SpectralTables& scan = s.scan32;
    double y = 0.0;
    for (size_t b = 0; b < kBins; ++b) {
        const double D = ((paper_d[0] * double(scan.eps[3 * b]) + paper_d[1] * double(scan.eps[3 * b + 1])) +
                          paper_d[2] * double(scan.eps[3 * b + 2])) +
                         double(scan.beta[b]);
        y += std::exp2(-D * kLog2Of10) * double(scan.wt[3 * b + 1]);
    }
    return std::max(y, 0.0) + 1e-10;
}

// scanner levels (reference src/print/setup.cpp:371-390): the line through the black and white targets of
// the print's Y at the film's extreme densities, and the exposure correction that keeps mid grey
void solve_levels(const PrintSetup& s, PrintRun& r) {
    const bool measured = !s.scanned && !s.paper_positive;
    if (measured) {
        r.y_k = printed_y(s, r, {-0.03, -0.03, -0.03});
        r.y_w = printed_y(s, r, s.film_white_density);
    }
    double black = s.levels_B, white = s.levels_W;
    if (s.levels_black && !s.levels_white) white = r.y_w;
    if (s.levels_white && !s.levels_black) black = r.y_k;
    r.m = (white - black) / (r.y_w - r.y_k + 1e-10);
    r.q = black - r.m * r.y_k;
    if (!measured) return;
    const Profile& paper = *s.paper;
    const double grey_level = (kMidGrey - r.q) / r.m;  // the Y that the line maps to mid grey
    const double e_target =
        interp(-std::log10(grey_level) - s.paper_mean_base, s.paper_mean_curve, paper.log_exposure);
    const double e_plain = interp(-std::log10(kMidGrey) - s.paper_mean_base, s.paper_mean_curve, paper.log_exposure);
    r.kappa_bw = std::pow(10.0, e_target - e_plain);
}

}  // namespace

PrintRun compute_run(const PrintSetup& s, const LiveParams& live) {
    PrintRun r;
    if (!s.scanned) {
        const Vec3 cc = {s.neutral[0], s.neutral[1] + live.m_filter_shift * live.filter_shift_scale,
                         s.neutral[2] + live.y_filter_shift * live.filter_shift_scale};
        r.light = enlarger_light(s.lamp, s.filters, cc);
        r.eps_n = s.film_eps;
        r.beta_n = s.film_beta;
        for (size_t b = 0; b < kBins; ++b)
            for (size_t c = 0; c < 3; ++c) r.w_n[3 * b + c] = r.light[b] * s.paper_sens[3 * b + c];
        drop_undefined_bins(r.eps_n, r.beta_n, r.w_n);
        const double phi = exposure_factor(s.compensation ? s.probe_comp : s.probe_mid, r.light, s.paper_sens);
        r.g = {phi, phi, phi};
        if (live.preflash_exposure > 0.0) {  // a flash through the film base alone, at the neutral filters
            const Vec3 e = layer_exposure(s.film_beta, enlarger_light(s.lamp, s.filters, s.neutral), s.paper_sens);
            for (size_t c = 0; c < 3; ++c) r.o[c] = live.preflash_exposure * e[c];
        }
    }
    r.levels = s.levels_active();
    if (r.levels) solve_levels(s, r);
    r.k_gain = f32(live.print_exposure * r.kappa_bw);
    to_f32(r.enl32.eps, r.eps_n);
    to_f32(r.enl32.beta, r.beta_n);
    to_f32(r.enl32.wt, r.w_n);
    return r;
}

}  // namespace spkb
