// The binary64 set-up of the render path: everything the kernels need that does not depend on a
// pixel, computed on the host once per pipeline build (film, print) or once per print (compute_run)
// and narrowed once to binary32. The floating-point expressions keep the operation order of the
// reference's set-up (src/film/setup.cpp, src/print/setup.cpp, src/print/build.cpp, src/print/cam16.cpp,
// src/fx/gaussian.cpp, src/fx/halation.cpp, src/fx/grain.cpp), so the narrowed constants equal the
// reference's bit for bit. Implemented in film_setup.cpp (blurs, grain, curves, couplers, the film
// set-up), upsampling.cpp (the spectral upsampling table), halation_setup.cpp, cam16.cpp and
// print_setup.cpp.
#pragma once

#include <array>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <string>
#include <vector>

#include "../kernel_args.h"
#include "params.hpp"
#include "resources.hpp"

namespace spkb {

// ---- Gaussian branch rule (reference src/fx/gaussian.hpp:6-15, gaussian.cpp:19-53) ----
enum class Branch { Identity, Fir, Iir };
Branch blur_branch(double sigma);                       // <= 0 identity, < 3 FIR, else recursive
int fir_radius(double sigma);                           // floor(3 sigma + 0.5)
std::vector<double> gaussian_kernel(double sigma, double truncate);  // normalised, ascending k
struct IirCoefficients {
    double B, B1, B2, B3;
};
IirCoefficients iir_coefficients(double sigma);         // Young and van Vliet 1995
// Their derivatives along sigma (B', B1', B2', B3'; the render's adjoint), from q'(sigma) and the
// quotient rule on b_i / b0.
IirCoefficients iir_coefficients_dsigma(double sigma);
// d/dsigma of the normalised FIR kernel on its fixed support: w_k (k^2 - sum_j w_j j^2) / sigma^3.
std::vector<double> gaussian_kernel_dsigma(double sigma, double truncate);

struct MixtureComponent {
    Vec3 weight;
    Vec3 sigma;  // pixels
};

// ---- halation (reference src/fx/halation.cpp:104-195) ----
struct HalationParams {
    bool active = true;
    double amount = 1.0, scatter_amount = 1.0, headroom_ev = 4.0;
    Vec3 scatter_core_um{2.2, 2.0, 1.6}, scatter_tail_um{9.3, 9.7, 9.1}, scatter_tail_weight{0.78, 0.65, 0.67};
    double scatter_scale = 1.0, halation_scale = 1.0;
    int bounces = 3;
    double bounce_decay = 0.5;
    bool renormalise = true;
    double base_thickness_um = 120.0;
    Vec3 strength{0.05, 0.015, 0.0};
    Vec3 first_sigma_um{65.0, 65.0, 65.0};
    bool back_reflection = false;
};
HalationParams resolve_halation(const Profile& film, const ParamSet& p);

struct HalationPlan {
    bool scatter = false;
    std::vector<MixtureComponent> scatter_comps;
    Vec3 scatter_a{}, scatter_b{};
    bool bounce = false;
    std::vector<MixtureComponent> bounce_comps;
    Vec3 mix_a{}, mix_b{};
};
HalationPlan halation_plan(const HalationParams& h, double pitch_um);

// A test and benchmark override of the bounce mixture: the components (sigma in pixels) and the
// strength A per channel, mixed as raw/(1 + A) + A H(raw)/(1 + A); the scatter stage is dropped.
struct HalationOverride {
    std::vector<MixtureComponent> comps;
    Vec3 strength{};
};

// ---- grain (reference src/fx/grain.cpp:66-152) ----
struct GrainSetup {
    bool active = false, sublayers = true, positive = false;
    double amount = 1.0;
    uint32_t K = 0;
    std::vector<float> axis, inv, layers;
    double f[3][3] = {}, dmin[3][3] = {}, sat_d[3][3] = {};
    double simple_d[3] = {};
};
struct GrainConstants {
    bool active = false, sublayers = true;
    double count[3][3] = {}, sat_d[3][3] = {}, dmin_l[3][3] = {}, sigma_dye[3][3] = {};
    bool dye = false, micro = false;
    double micro_sigma = 0, micro_blur = 0, final_blur = 0;
};
GrainConstants grain_constants(const GrainSetup& g, double pitch_um);
// An exponential PSF of scale lambda_px as three Gaussians of total weight `weight`.
std::array<MixtureComponent, 3> exponential_surrogate(const Vec3& weight, const Vec3& lambda_px);
inline constexpr double kGrainDmin[3] = {0.03, 0.03, 0.03};

// ---- film set-up (reference src/film/setup.cpp:353-419) ----
struct FilmSetup {
    ParamSet params;
    std::shared_ptr<const Profile> profile;
    bool positive = false;
    ColourSpace input_space;
    bool decode = false;          // input_cctf_decoding: the input space's transfer function is undone first
    std::array<double, 2> illuminant_xy{};
    Mat3 input_matrix{};
    std::array<float, 9> input_matrix_f32{};
    uint32_t L = 0;
    std::vector<double> table64;  // L x L x 3
    std::vector<float> table32;
    HalationParams halation;
    std::shared_ptr<GrainSetup> grain;
    uint32_t K = 0;
    std::vector<float> cx, cinv, cy, cy0;  // curve tables, y channel-major
    // DIR couplers (reference src/film/setup.cpp:25-95, :402-406): the coupler matrix M[donor][receiver],
    // the stock's D_max, and the pre-inverted curve y0 (cy0; binary64 in cy0_64, channel-major)
    bool couplers = false;
    Mat3 coupler_m{};
    std::array<float, 9> coupler_m_f32{};
    Vec3 dmax{};
    std::array<float, 3> dmax_f32{};
    std::vector<double> cy0_64;
};
std::shared_ptr<FilmSetup> build_film_setup(const ParamSet& p, std::shared_ptr<const Profile> film,
                                            const Resources& res);
// The L x L x 3 spectral upsampling table (upsampling.cpp; reference src/film/setup.cpp:133-257): the layer
// sensitivities sens (bin-major, shaped by the stock's adaptation window under `light`) contracted with
// every grid node's spectrum, read back at the node's gamut-compressed chromaticity.
std::vector<double> spectral_upsampling_table(const Blob& blob, const std::array<double, 243>& sens,
                                              const std::vector<double>& window, const Spectrum& light,
                                              uint32_t* L_out);

// ---- CAM16-UCS (reference src/print/cam16.cpp) ----
struct Cam16Constants {
    double L_A = 64.0, Y_b = 20.0, F = 1.0, c = 0.69, N_c = 1.0, Y_w = 100.0;
    double n = 0, k = 0, F_L = 0, N_bb = 0, N_cb = 0, z = 0, D = 0;
    Vec3 rgb_w{}, D_rgb{};
    double A_w = 0, J_white = 0;
    Mat3 m16{}, m16_inv{};
};
Cam16Constants cam16_constants(const std::array<double, 2>& wp);
struct Cam16Forward {
    double J, C, h, M, Jp, Mp;
};
Cam16Forward cam16_forward(const Cam16Constants& k, const Vec3& xyz);
Vec3 cam16_inverse_unguarded(const Cam16Constants& k, double Jp, double ap, double bp);
std::vector<double> cam16_cmax_table(const Cam16Constants& k, const Mat3& m_to_rgb);  // 64 x 720

struct Cam16Tables {
    std::string space;
    Cam16Constants k;
    Mat3 m_to_xyz{}, m_to_rgb{};
    std::vector<double> cmax64;
    std::vector<float> cmax32;
};

// ---- print set-up (reference src/print/build.cpp:53-236, src/print/setup.cpp) ----
struct LiveParams {
    double print_exposure = 1.0, m_filter_shift = 0.0, y_filter_shift = 0.0, preflash_exposure = 0.0,
           filter_shift_scale = 1.0;
    static LiveParams from(const ParamSet& p);
};

struct PrintSetup {
    ParamSet params;
    std::shared_ptr<const Profile> paper;
    ColourSpace out_cs;
    bool scanned = false, compensation = true;
    Spectrum lamp{};
    std::array<Spectrum, 3> filters{};
    Vec3 neutral{};
    std::array<double, 243> paper_sens{}, film_eps{};
    Spectrum film_beta{}, probe_mid{}, probe_comp{};
    uint32_t paper_K = 0;
    std::vector<float> paper_tab;  // x[K], r[K], y[K][3]
    std::vector<double> paper_y64;  // the cdfs curve before narrowing, K x 3
    std::array<double, 243> scan_eps{}, scan_wt{};
    Spectrum scan_beta{};
    Vec3 view_xyz{};
    SpectralTables scan32{};
    Mat3 to_rgb64{}, m_nid64{};
    float to_rgb[9] = {};
    std::shared_ptr<const Cam16Tables> cam;
    Cam16Args cam_args{};
    bool cctf = true;
    float m_nid[9] = {};
    uint32_t cctf_mode = 1;
    double scanner_lens_blur_px = 0.0, unsharp_sigma_full = 0.7, unsharp_amount = 0.7;
    // print glare (reference src/fx/glare.hpp:13-20): percent 0.03, roughness 0.7, blur 0.5 px at the full
    // tier, tinted by the viewing illuminant's XYZ at Y = 1
    bool glare = false;
    double glare_amount = 1.0, glare_percent = 0.03, glare_roughness = 0.7, glare_blur_full = 0.5;
    Vec3 glare_tint{};
    bool glare_draws() const { return glare && glare_percent * glare_amount > 0.0; }
    // scanner levels (reference src/print/build.cpp:152-155, src/print/setup.cpp:262-270): black and
    // white targets B and W, the film's white density, the paper's mean curve and base for the exposure
    // correction; a directly scanned negative passes through
    bool levels_black = false, levels_white = false, film_positive = false, paper_positive = false;
    double levels_B = 0.0, levels_W = 0.0, paper_mean_base = 0.0;
    Vec3 film_white_density{};
    std::vector<double> paper_mean_curve;
    // the EDR tone map (reference src/print/build.cpp:83-85, :210-222), from the paper profile
    bool edr = false;
    double edr_lo = 0.0, edr_hi = 0.0, edr_toe = 0.0, edr_shoulder = 0.0;
    std::vector<float> edr_tab;
    bool levels_active() const {
        if (!levels_black && !levels_white) return false;
        return scanned ? film_positive : true;
    }
};

class Cam16Cache {
public:
    std::shared_ptr<const Cam16Tables> get(const Resources& res, const std::string& space);

private:
    std::mutex m_;
    std::map<std::string, std::shared_ptr<const Cam16Tables>> by_space_;
};

std::shared_ptr<PrintSetup> build_print_setup(const ParamSet& p, const FilmSetup& film,
                                              std::shared_ptr<const Profile> paper, const Resources& res,
                                              Cam16Cache& cache, bool compensation);

// The per-print constants (reference src/print/setup.cpp:339-399).
struct PrintRun {
    Spectrum light{};
    std::array<double, 243> eps_n{}, w_n{};
    Spectrum beta_n{};
    Vec3 g{}, o{};
    float k_gain = 1.0f;
    SpectralTables enl32{};
    bool levels = false;
    double m = 1.0, q = 0.0, y_k = 0.0, y_w = 1.0, kappa_bw = 1.0;
};
PrintRun compute_run(const PrintSetup& s, const LiveParams& live);

// Mitchell-Netravali (B = C = 1/3) sample of an L x L x 3 table, binary64 (reference src/print/setup.cpp:148-160).
Vec3 bicubic_sample(const std::vector<double>& table, uint32_t L, double t0, double t1);

}  // namespace spkb
