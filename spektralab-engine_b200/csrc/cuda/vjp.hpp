// The adjoint (vector-Jacobian product) of the render path: kernels of vjp.cu and their arguments.
//
// The differentiated output is the scanned linear RGB (the scanner's lens blur and unsharp mask applied,
// before the output transfer function and the 16-bit encode), with the grain held as fixed noise (the
// Poisson counts of one film seed). The per-pixel stages run on dual numbers (dual.cuh); the blurs take
// their exact transposes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"

namespace spkb::dev {

constexpr int kVjpPrintParams = 3;  // print_exposure, m_filter_shift, y_filter_shift
// Density-curve parameters: per film layer c, 16 hat functions on the entries of its K-entry curve table,
// phi_j(k) = max(0, 1 - |u_k - j|) with u_k = 15 k / (K - 1). theta[c][j] adds theta phi_j(k) to every entry
// y_c[k], so the lookup's linear interpolation gives dD/dtheta_j = (1 - t) phi_j(l) + t phi_j(l + 1).
constexpr int kVjpCurveNodes = 16;

// The print stage in the adjoint's form: the set-up's narrowed tables as they are (no packing), and the
// tangents of the enlarger tables and gains along each print-side parameter (formed on the host by
// central differences of the binary64 set-up; zero where a table does not depend on the parameter).
struct VjpPrintArgs {
    float enl_eps[SPKB_NL * 3], enl_beta[SPKB_NL], enl_wt[SPKB_NL * 3];
    float t_eps[kVjpPrintParams][SPKB_NL * 3], t_beta[kVjpPrintParams][SPKB_NL], t_wt[kVjpPrintParams][SPKB_NL * 3];
    float g[3], o[3], k_gain;
    float t_g[kVjpPrintParams][3], t_o[kVjpPrintParams][3], t_k[kVjpPrintParams];
    float scan_eps[SPKB_NL * 3], scan_beta[SPKB_NL], scan_wt[SPKB_NL * 3];
    int32_t printed;
    const float* paper;  // x[K], r[K], y[K][3]
    uint32_t paper_K;
    AxisGrid paper_grid;
    float to_rgb[9];
    Cam16Args cam;
    const float* cmax;
    uint32_t n;
};

// g_neg = J^T g_P per pixel of the print stage (negative -> linear output RGB); grad_params[j] += the
// sum over pixels of g_P . dP/dparam_j (binary64 accumulation).
void vjp_print(const float* neg, const float* g_print, float* g_neg, double* grad_params, const VjpPrintArgs& a,
               cudaStream_t s);

// g_exposure = J^T g_neg per pixel and channel of the develop stage: log10, density curve, sub-layer
// densities and the grain value with the counts held fixed (counts: 9 floats per pixel [c][l]).
// g_nodes (may be null): g_nodes[c * 16 + j] += the sum over pixels of g_neg_c dneg_c/dtheta[c][j]
// (binary64 accumulation).
void vjp_develop(const float* exposure, const float* counts, const float* g_neg, float* g_exposure,
                 double* g_nodes, const DevelopArgs& a, uint32_t w, uint32_t h, cudaStream_t s);

// g_rgb = J^T g_h per pixel of the expose stage (RGB -> film exposure through the spectral table).
void vjp_expose(const float* rgb, const float* g_h, float* g_rgb, const float* table4, const ExposeArgs& a,
                cudaStream_t s);

// The transpose of one pass of the engine's FIR (taps[0..2r], half-sample symmetric reflection at the
// edges; vertical != 0: along columns): g_in := pass^T g_out.
void fir_pass_adjoint(const float* g_out, float* g_in, uint32_t w, uint32_t h, int r, const float* taps,
                      int vertical, cudaStream_t s);

// acc[c] += sum over pixels of x[i] y[i] for each channel c = i % 3 (binary64)
void dot3(const float* x, const float* y, size_t pixels, double* acc, cudaStream_t s);

}  // namespace spkb::dev
