/* Test infrastructure: the float64 oracle of the spektralab render path.
 *
 * A CPU restatement, in binary64, of the reference engine's per-pixel render path: every stage of
 * the film side (src/film/develop.cpp:101-236) and the print side (src/print/run.cpp:118-188) with
 * the reference kernels' formulas (kernels/*.metal) evaluated in double, fed from the unrounded
 * binary64 set-up. Only the tests, the smoke check and the benchmark's CPU baseline load it; the
 * product never does. Its own correctness is pinned against the reference engine run on this CPU
 * (oracle/_ref) and the golden vectors in tests/golden.
 *
 * Grain: the Poisson counts are either drawn here with the binary32 sampler shared with the device
 * code (grain_sampler.h) from lambda rounded to binary32, or taken from the caller ("fixed noise"),
 * so that a device render can be compared with the float64 arithmetic of every other stage.
 */
#ifndef SPK_ORACLE_H
#define SPK_ORACLE_H

#include <stdint.h>

#define ORC_MAX_COMP 8

typedef struct {
    /* expose */
    double A[9];
    double gain;
    int32_t L;
    const double* table; /* L*L*3 */
    /* halation: scatter mixture then bounce mixture, each raw := a raw + b M(raw) */
    int32_t n_scatter, n_bounce;
    double scatter_w[ORC_MAX_COMP][3], scatter_s[ORC_MAX_COMP][3], scatter_a[3], scatter_b[3];
    double bounce_w[ORC_MAX_COMP][3], bounce_s[ORC_MAX_COMP][3], mix_a[3], mix_b[3];
    double lens_blur_px;
    /* curves */
    int32_t K;
    const double* cx;
    const double* cinv;
    const double* cy; /* 3K, channel-major */
    /* grain */
    int32_t grain, positive, gK;
    const double* gaxis;   /* K*3 */
    const double* ginv;    /* K*3 */
    const double* glayers; /* K*3*3 */
    double count[9], sat_d[9], dmin_l[9], uniformity[3], dmin_c[3];
    double final_blur, amount;
    uint32_t seed;
    /* print */
    int32_t printed;
    double enl_eps[243], enl_beta[81], enl_wt[243], g[3], o[3], k_gain;
    int32_t pK;
    const double* px;
    const double* pr;
    const double* py; /* pK*3 */
    double scan_eps[243], scan_beta[81], scan_wt[243];
    double to_rgb[9];
    /* CAM16 gamut */
    double cam_k[22]; /* F_L N_bb N_cb n z A_w c N_c Jfirst Jlast hfirst hstep knee0..2 lc0..2 Jwhite D_R D_G D_B */
    double m_to_xyz[9], m_to_rgb[9], m16[9], m16_inv[9];
    const double* cmax; /* 64 x 720 */
    int32_t lc_active;
    /* scanner + encode */
    double scanner_lens_blur, unsharp_sigma, unsharp_amount;
    int32_t cctf_active, cctf_mode;
    double m_nid[9];
    /* DIR couplers (reference src/film/develop.cpp:203-226): chi_m := sum_c s_c M[c][m] with
     * s := positive ? dmax - D : D from the first development D, chi := sum_k dir_w[k] G(dir_s[k]) chi,
     * then the density is the pre-inverted curve cy0 at log10 exposure - chi */
    int32_t couplers, n_dir;
    double coupler_m[9], dmax[3];
    const double* cy0; /* 3K, channel-major */
    double dir_w[ORC_MAX_COMP][3], dir_s[ORC_MAX_COMP][3];
    /* print glare (reference src/fx/glare.cpp:27-50): a lognormal field (binary32 mean and sd, stream 200,
     * the print seed) blurred by glare_sigma and added to the scan's XYZ as (F / 100) tint */
    int32_t glare;
    float glare_mean, glare_sd;
    double glare_sigma, glare_tint[3];
    uint32_t print_seed;
    /* the highlight boost (boost_ev != 0) and the back-reflection headroom (headroom_ev > 0 when it applies),
     * both on the exposure after the compensation, against the frame maximum */
    double boost_ev, headroom_ev;
    /* scanner levels on the scan's XYZ before the glare: Y' = clamp(m Y + q, 0, 1), XYZ times Y' / (Y + 1e-10) */
    int32_t levels;
    double levels_m, levels_q;
    /* the EDR tone map after the scanner: y = max(r_y . rgb, 0); outside [toe, shoulder] y' = 2^(the target
     * curve at the clamped (log2 y - lo) / (hi - lo)); rgb times y' / (y + 1e-10) */
    int32_t edr, edr_n;
    double edr_r_y[3], edr_lo, edr_hi, edr_toe, edr_shoulder;
    const double* edr_tab;
} OracleSetup;

/* The whole render of a w x h frame; rgb is 3 floats per pixel (already non-finite-cleaned),
 * counts NULL or 9 floats per pixel [c][l]; out_rgba receives w*h*4 uint16 (packed rows),
 * out_negative (may be NULL) w*h*3 doubles. Returns 0. */
int orc_render(const OracleSetup* s, const float* rgb, int32_t w, int32_t h, const float* counts,
               uint16_t* out_rgba, double* out_negative);

/* Film side only / print side only (the print side of a given negative, for reprints). */
int orc_develop(const OracleSetup* s, const float* rgb, int32_t w, int32_t h, const float* counts, double* negative);
int orc_print(const OracleSetup* s, const double* negative, int32_t w, int32_t h, uint16_t* out_rgba,
              double* out_linear_rgb);

/* The scanned linear RGB (print, scanner lens blur and unsharp mask, before the transfer function and
 * the encode) of a binary64 frame, for the finite-difference checks of the render's adjoint; counts as
 * for orc_render. Returns 0. */
int orc_render_linear(const OracleSetup* s, const double* rgb, int32_t w, int32_t h, const float* counts,
                      double* out_linear);

/* The print's spectral integral (reference kernels/print.metal:165-189) at nl wavelengths for n pixels:
 * out[p][k] = sum_l 10^-(sum_c d[p][c] eps[l][c] + beta[l]) wt[l][k], binary64, ascending l. */
void orc_spectral(const double* eps, const double* beta, const double* wt, int32_t nl, const double* d, int64_t n,
                  double* out);

/* The Gaussian of a w x h x 3 plane, per-channel sigma in pixels, in binary64 with the engine's
 * branch rule (FIR below 3, Young-van Vliet above) */
void orc_gaussian(const double* in, double* out, int32_t w, int32_t h, const double sigma[3]);

/* The tier downscale (reference src/session/tiers.cpp:99-227, session.metal:19-91), restated in the
 * binary32 arithmetic that the reference specifies for both its GPU and CPU paths (taps narrowed from
 * binary64, fmaf in ascending tap order, mirror edges, exact-integer bilinear tables), so that every
 * implementation gives the same bits: src w x h x 3 -> dst ow x oh x 3. Returns 0. */
int orc_downscale(const float* src, int32_t w, int32_t h, int32_t ow, int32_t oh, float* dst);

/* The input transfer decode (reference kernels/film.metal:104-142; mode 0 sRGB, 1 ProPhoto, 2 Adobe,
 * 3 BT.709, 4 identity; decode = 0 skips it) and the crop / rotation / quarter turn / flip geometry
 * (src/film/geometry.cpp:45-157: geo = {crop_x, crop_y, crop_w, crop_h, rotation_deg, quarter_turns,
 * flip_h, flip_v}), both in binary64: src w x h x 3 -> dst of the geometry's output size, written to
 * *ow, *oh (dst holds at least w h 3 doubles: the crop never exceeds the frame). Returns 0. */
int orc_prepare(const float* src, int32_t w, int32_t h, int32_t decode, int32_t mode, const double geo[8],
                double* dst, int32_t* ow, int32_t* oh);

/* The auto-exposure meter (reference src/film/meter.cpp:45-120) of a binary64 image, in binary64:
 * Y = row 1 of rgb_to_xyz . rgb; out = {center_weighted, average, median, balanced, center,
 * protect_highlights, protect_shadows}. Returns 0. */
int orc_meter(const double* rgb, int32_t w, int32_t h, const double rgb_to_xyz[9], double out[7]);

/* orc_render on a binary64 frame (the output of orc_prepare). */
int orc_render64(const OracleSetup* s, const double* rgb, int32_t w, int32_t h, const float* counts,
                 uint16_t* out_rgba, double* out_negative);

/* The shared binary32 sampler (grain_sampler.h), for the bit-exactness tests. */
void orc_poisson(const float* lam, float* counts, uint32_t n, uint32_t stream, uint32_t seed);
void orc_lognormal(float* out, uint32_t n, float mean, float sd, uint32_t stream, uint32_t seed);
void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out, uint32_t n);
float orc_uniform(uint32_t word);
float orc_logf(float x);
float orc_expf(float x);
float orc_cosf(float x);
uint32_t orc_splitmix_next(uint64_t* state);

#endif
