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
    uint32_t L;        // table size; the table is L x L x 3, [i][j][c]
    uint32_t n;        // pixels
};

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

// Film-side point work after halation: log10 exposure, density curves, grain draw.
struct DevelopArgs {
    // curves: x[K], inv[K], y[3K] (channel-major)
    const float* cx;
    const float* cinv;
    const float* cy;
    uint32_t K;
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
    float uniformity[3];
    float dmin_c[3];
    const float* axis;    // [k*3 + c]
    const float* ginv;    // [k*3 + c]
    const float* layers;  // [(k*3 + l)*3 + c]
    uint32_t width;       // pixel index = y * width + x keys the draws
    float* counts_out;    // test hook: the Poisson counts, [pixel][c][l]; nullptr in renders
};

// Per-wavelength tables of one spectral integral (already neutralised).
struct SpectralTables {
    float eps[SPKB_NL * 3];  // [l][c]
    float beta[SPKB_NL];
    float wt[SPKB_NL * 3];   // [l][k]
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
};

// The print kernel: negative density -> linear output RGB.
struct PrintArgs {
    SpectralTables enl;
    SpectralTables scan;
    float g[3], o[3];
    float k_gain;
    int32_t printed;            // 0: scan_film (the negative is scanned directly)
    const float* paper;         // x[K], r[K], y[K][3]
    uint32_t paper_K;
    float to_rgb[9];
    Cam16Args cam;
    const float* cmax;
    uint32_t n;
};

// Scanner unsharp + transfer function + 16-bit encode.
struct EncodeArgs {
    float m_nid[9];
    int32_t cctf_active;
    uint32_t cctf_mode;   // 0 sRGB, 1 ProPhoto, 2 Adobe, 3 BT.709, 4 identity
    uint32_t stride;      // output row pitch in pixels
    float lincomb_a, lincomb_b;  // out = a x + b g (unsharp), applied when unsharp != 0
    int32_t unsharp;
};
