// Argument records shared by the host set-up (C++) and the sm_100a kernels (CUDA).
//
// Every record is plain data passed by value to a kernel (__grid_constant__), so the per-wavelength
// tables sit in the kernel's constant bank and a warp-uniform loop over wavelength reads them by
// broadcast. The float values are the host's binary64 set-up narrowed once (round to nearest).
#pragma once

#include <stdint.h>

#define SPKB_NL 81          // wavelength samples, 380..780 nm at 5 nm
#define SPKB_FIR_MAX_R 9    // FIR branch: sigma < 3 gives R = floor(3 sigma + 0.5) <= 9
#define SPKB_MAX_COMPONENTS 8

// Spectral upsampling + exposure compensation (the expose pass).
struct ExposeArgs {
    float a[9];        // input matrix A, row-major
    float gain;        // f32(2^exposure_compensation_ev)
    int32_t apply_gain;
    float ae_gain;     // f32(2^ev) of the auto-exposure meter, on the RGB before the upsampling
    int32_t apply_ae;
    uint32_t L;        // table size; the table is L x L float4 texels, [i][j] = (R, G, B, 0)
    uint32_t n;        // pixels
};
// floats of one 4 x 4 patch of the spectral table (16 RGB texels)
#define kPatchFloats 48u

// One separable FIR Gaussian: taps -r..r per channel (a channel without a FIR blur holds the delta).
struct FirTaps {
    int32_t r;
    float taps[3][2 * SPKB_FIR_MAX_R + 1];
};

// One recursive (Young-van Vliet) Gaussian: binary64 coefficients per channel; mask bit c set when
// channel c is filtered (the others pass through unchanged).
struct IirCoefs {
    uint32_t mask;
    double B[3], B1[3], B2[3], B3[3];
};

// Accumulation of a blur's last pass: out = v, out = 0 + w v, or out = acc + w v.
enum AccMode { ACC_NONE = 0, ACC_ZERO = 1, ACC_PLANE = 2 };

// Direct index into an ascending binary32 axis x[0..K-1]: g(v) = clamp(int((v - x0) s), 0, K - 2). The
// host sets `active` only after checking that g is within one of the bisection's interval for every v
// in (x[0], x[K-1]); the kernel then corrects g by one comparison on each side. Inactive: bisection.
struct AxisGrid {
    float x0, s;
    int32_t active;
};

// Film-side point work after halation: log10 exposure, density curves, grain draw.
struct DevelopArgs {
    // curves: x[K], inv[K], y[3K] (channel-major)
    const float* cx;
    const float* cinv;
    const float* cy;
    uint32_t K;
    AxisGrid cgrid;       // the curves' log-exposure axis
    AxisGrid ggrid[3];    // the grain layers' density axis of each channel
    // grain (reference fx_grain.metal:39-97 modes)
    int32_t grain;        // 0: no grain, write the density
    uint32_t mode;        // 0 SUM (sub-layers, no dye clouds), 1 PLANES, 2 SIMPLE
    uint32_t seed;
    uint32_t gK;          // grain axis points
    uint32_t positive;
    uint32_t shift;       // subtract D_min,c in the draw
    uint32_t n_sub;
    float inv_n_sub;
    float dmin_l[9], sat_d[9], count[9];
    float unit[9];        // sat_d / count, the binary32 quotient (a draw's density per grain before saturation)
    float uniformity[3];
    float dmin_c[3];
    const float* axis;    // [k*3 + c]
    const float* ginv;    // [k*3 + c]
    const float* layers;  // [(k*3 + l)*3 + c]
    uint32_t width;       // pixel index = y * width + x keys the draws
    float* counts_out;    // test hook: the Poisson counts, [pixel][c][l]; nullptr in renders
    float* lam_out;       // test hook: the draws' lambdas, [pixel][c][l] (sub-layer grain); nullptr in renders
    // DIR couplers: the blurred correction plane chi (interleaved RGB), subtracted from the log exposure
    // before the curve lookup, with cy then the pre-inverted curve y0; nullptr without couplers
    const float* chi;
};

// DIR couplers' source (reference kernels/film.metal:242-276): the first development of the exposure
// through the density curve (x, inv, y), then chi_m = sum_c s_c M[c][m], s_c = positive ? dmax_c - D_c : D_c.
struct CouplerArgs {
    const float* cx;
    const float* cinv;
    const float* cy;
    uint32_t K;
    AxisGrid cgrid;
    uint32_t positive;
    float m[9];           // M[c * 3 + m], c the donor layer
    float dmax[3];
    uint32_t n;           // pixels
};

// Tier downscale (reference src/session/tiers.cpp:137-183, kernels/session.metal:19-91): a vertical
// Gaussian prefilter over the frame (k_tier_blur_v), then one pass per output pixel that evaluates the
// horizontal prefilter at the four points its bilinear sample reads and blends them. Mirror edges,
// taps -r..r ascending, acc = fma(w_k, x, acc) from 0; the index tables are the host's exact integers.
struct TierBlurArgs {
    const float* taps;  // 2 r + 1
    uint32_t w, h;
    int32_t r;          // >= 1
};
struct TierResampleArgs {
    const float* taps_x;  // 2 rx + 1 (rx = 0: no horizontal prefilter)
    const uint32_t* xi;   // [2 out_w]: i0, i1
    const float* xt;      // [out_w]
    const uint32_t* yi;   // [2 out_h]
    const float* yt;      // [out_h]
    uint32_t in_w, in_h, out_w, out_h;
    int32_t rx;
};

// Input transfer decode and geometry (reference kernels/film.metal:104-173, src/film/geometry.cpp:45-107)
// in one pass over the output: each bilinear tap is decoded before the blend, which gives the values of
// the decode pass followed by the geometry pass. The kernel forms the plan's binary64 column and row
// terms itself, by the host plan's operations (no contraction), and splits them into two binary32 as the
// reference's host does before its launch.
struct PrepareArgs {
    int32_t decode;         // 0: the input is linear
    uint32_t mode;          // transfer function: 0 sRGB, 1 ProPhoto, 2 Adobe, 3 BT.709, 4 identity
    float bt709_bp, bt709_exp;
    int32_t geometry;       // 0: identity (dst = decoded src, same size)
    uint32_t quarter, flip_h, flip_v;
    uint32_t src_w, src_h, dst_w, dst_h;
    double sx, sy, hx, hy;  // per-axis scale and half extent of the crop, in source pixels
    double ca, sa;          // cos and sin of the rotation
    double ow, oh;          // the output size
    double cx, cy;          // the crop centre in source pixel coordinates
};

// The auto-exposure meter's device statistics (reference src/film/meter.cpp:45-120). Six order-statistic
// queries on the ascending luminances (NaN last): the two middle ranks (the same rank twice for an odd
// count), then the ranks q (n - 1) / 1000 for q = 10, 50, 990, 995.
#define kMeterQueries 6
#define kMeterMedLo 0
#define kMeterMedHi 1
#define kMeterP10 2
#define kMeterP50 3
#define kMeterP990 4
#define kMeterP995 5
struct MeterSelect {
    uint64_t rank[kMeterQueries];    // the rank still to find inside the current prefix
    uint64_t prefix[kMeterQueries];  // the ordered key's digits found so far
    uint64_t mask[kMeterQueries];
    uint32_t hist[kMeterQueries][256];
    double value[kMeterQueries];     // the selected luminances
};
struct MeterOut {
    // sum Y, sum w Y, sum w; then over the intent range: sum ln y, sum w ln y, sum w, count
    double sums[7];
    double select[kMeterQueries];
};
struct MeterArgs {
    const float* rgb;   // the meter image, interleaved RGB
    uint32_t w, h;
    uint64_t n;
    double m0, m1, m2;  // row Y of the input space's RGB -> XYZ matrix
    uint64_t* key;      // n ordered keys (scratch)
    double* partial;    // 7 x the launch's blocks (scratch)
    MeterSelect* sel;
    MeterOut* out;
};

// The print-preview table render (reference kernels/print.metal:368-407): per pixel the negative's
// densities through a trilinear S x S x S x 3 table, then the 16-bit encode.
struct PrintLutArgs {
    const float* lut;   // [i][j][k][ch], row-major
    uint32_t size;      // S
    uint32_t w, h, stride;  // output row pitch in pixels
    float lo[3], s[3];  // axis start and f32(1 / (hi - lo)) per channel
};

// Per-wavelength tables of one spectral integral (already neutralised).
struct SpectralTables {
    float eps[SPKB_NL * 3];  // [l][c]
    float beta[SPKB_NL];
    float wt[SPKB_NL * 3];   // [l][k]
};

// One spectral integral in the print kernel's form, for packed f32x2 arithmetic over a pair of pixels:
// e_c(l) = -log2(10) eps_c(l) and w_k(l) = wt_k(l) 10^-beta(l), each value held twice (both halves of a
// packed operand), so that sum_l 2^(sum_c d_c e_c(l)) w_k(l) = sum_l 10^-D(l) wt_k(l).
struct alignas(8) F32Pair {
    float x, y;
};
struct SpectralPairs {
    F32Pair e[SPKB_NL * 3];  // [l][c]
    F32Pair w[SPKB_NL * 3];  // [l][k]
};

// The arithmetic of the print's two spectral integrals in the spectral-mode print kernel
// (k_print_spectral): binary32 or binary64 on the CUDA cores, or the sum over wavelengths on the tensor
// cores (tcgen05) with binary32 accumulation: TF32 operands, BF16 operands, or BF16 hi + lo splits of
// both operands (T w = (Th + Tl)(wh + wl), four products).
#define SPKB_NL_MAX 416  // wavelength samples of the spectral-mode kernel: 401 (1 nm) padded to 32
enum SpectralMode : int32_t {
    SPKB_SPEC_F32 = 0,
    SPKB_SPEC_F64 = 1,
    SPKB_SPEC_TF32 = 2,
    SPKB_SPEC_BF16 = 3,
    SPKB_SPEC_BF16X3 = 4,
};

// The print's two spectral integrals at nl wavelengths for the spectral-mode kernel, in device memory.
// Pass 0 is the enlarger (film densities -> print exposure), pass 1 the scan (print densities -> XYZ);
// in both, R_k = sum_l 2^(sum_c d_c e_c(l)) w_k(l) with e_c = -log2(10) eps_c and w_k = wt_k 10^-beta.
// Every table is zero from nl to nl_pad.
struct SpectralTablesN {
    uint32_t nl, nl_pad;  // nl_pad: nl rounded up to a multiple of 32
    uint32_t pad_[2];
    // e in wavelength pairs: [pass][l / 2] = {e0(l), e0(l+1), e1(l), e1(l+1), e2(l), e2(l+1), 0, 0}
    float e_pairs[2][SPKB_NL_MAX / 2][8];
    float w[2][SPKB_NL_MAX][4];    // [pass][l] = {w0, w1, w2, 0}
    double e64[2][SPKB_NL_MAX][4];  // the binary64 values, before narrowing
    double w64[2][SPKB_NL_MAX][4];
    // The tensor cores' B operand of each pass: 16 rows n by nl_pad columns l, K-major without swizzle:
    // element (n, l) at byte ((n / 8) * (nl_pad * S / 16) + (l * S) / 16) * 128 + (n % 8) * 16 + (l * S) % 16,
    // S the element size (8-row by 16-byte core matrices, the K direction's fastest).
    //   bf16: rows 0..2 bf16(w_k), rows 3..5 bf16(w_k - bf16(w_k)), rows 6..15 zero;
    //   tf32: rows 0..2 w_k (binary32; the tensor core reads its TF32 part), rows 3..15 zero.
    uint16_t b_bf16[2][16 * SPKB_NL_MAX];
    float b_tf32[2][16 * SPKB_NL_MAX];
};

// CAM16-UCS gamut compression constants (reference kernels/print_shared.h:74-100 field meanings).
struct Cam16Args {
    uint32_t rows, cols;
    float m_to_xyz[9], m_to_rgb[9], m16[9], m16_inv[9];
    float d_rgb[3];
    float f_l, n_bb, n_cb, n, z, a_w, c, n_c;
    float j_first, j_last, h_first, h_step;
    float knee[3], lc[3];
    uint32_t lc_active;
    float j_white;
    // per-frame constants of the reference's per-pixel set-up (kernels/print.metal:53-64), formed on the
    // host in binary32 by the same operations: c z, 1 / (c z), F_L^0.25, (1.64 - 0.29^n)^0.73, 100 / F_L
    float cz, inv_cz, f_l_qrt, chroma_k, hundred_over_f_l;
    // binary32 reciprocals of the frame's divisors, for the gamut stage's approximate arithmetic
    float inv_a_w, inv_j_white, inv_n_bb, inv_f_l_qrt, inv_h_step, inv_j_span, inv_d_rgb[3];
    float knee_inv_span, knee_inv_p, lc_inv_span, lc_inv_p;  // 1 / (lim - tau), 1 / p of the two knees
};

// The print kernel: negative density -> linear output RGB.
struct alignas(16) PrintArgs {
    SpectralPairs enl;
    SpectralPairs scan;
    float g[3], o[3];
    float k_gain;
    int32_t printed;            // 0: scan_film (the negative is scanned directly)
    const float* paper;         // x[K], r[K], y[K][3]
    uint32_t paper_K;
    AxisGrid paper_grid;
    float to_rgb[9];
    Cam16Args cam;
    const float* cmax;
    uint32_t n;
    // print glare: the blurred lognormal field (interleaved RGB, equal channels), added to the scan's XYZ
    // as (F / 100) tint before the output matrix; nullptr without glare
    const float* glare;
    float glare_tint[3];
    // scanner levels (reference kernels/print.metal:234-246): Y' = clamp(m Y + q, 0, 1), XYZ times
    // Y' / (Y + 1e-10), before the glare; levels = 0: none
    int32_t levels;
    float levels_m, levels_q;
};

// Scanner unsharp + transfer function + 16-bit encode.
struct EncodeArgs {
    float m_nid[9];
    int32_t cctf_active;
    uint32_t cctf_mode;   // 0 sRGB, 1 ProPhoto, 2 Adobe, 3 BT.709, 4 identity
    uint32_t stride;      // output row pitch in pixels
    float lincomb_a, lincomb_b;  // out = a x + b g (unsharp), applied when unsharp != 0
    int32_t unsharp;
    // the EDR tone map on luminance (reference kernels/print.metal:319-347), after the unsharp mask and
    // before the output matrix; edr = 0: none
    int32_t edr;
    uint32_t edr_n;             // target_log2_y points
    float edr_r_y[3];           // row Y of the output space's RGB -> XYZ
    float edr_lo, edr_span, edr_toe, edr_shoulder;
    const float* edr_tab;       // target_log2_y, binary32
};

// The scanner's two FIR blurs, the unsharp combine and the encode in one tiled pass
// (reference src/fx/scanner.cpp:16-31 and kernels/print.metal:350-366). Both blurs have one sigma for
// all three channels, so one tap vector each; r = 0 with taps {1} is the identity.
struct ScanArgs {
    int32_t r1;                              // lens blur radius
    float t1[2 * SPKB_FIR_MAX_R + 1];
    int32_t r2;                              // unsharp blur radius (0 when unsharp is off)
    float t2[2 * SPKB_FIR_MAX_R + 1];
    EncodeArgs e;
};

// One frame of a batched print launch (k_print_batch): its arguments and planes.
struct alignas(16) BatchPrintFrame {
    PrintArgs args;
    const float* neg;
    float* rgb;
};

// One frame of a batched scanner launch (k_scan_encode_batch): its tiles are first_tile ..
// first_tile + tiles_x * tiles_y - 1 of the launch's tile list.
struct BatchScanFrame {
    ScanArgs args;
    const float* rgb;
    uint16_t* out;
    uint32_t w, h, tiles_x, first_tile;
};
