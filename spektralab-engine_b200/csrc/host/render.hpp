// The render path on the device: film side (develop) and print side (print, scan, encode), driven
// from the binary64 set-up. Stage order and the rules of every blur follow the reference
// (src/film/develop.cpp:101-236, src/print/run.cpp:118-188, src/fx/gaussian.cpp:167-273,
// src/fx/halation.cpp:307-329, src/fx/grain.cpp:167-267, src/fx/scanner.cpp:16-31); the kernels are
// this build's own (csrc/cuda).
#pragma once

#include <cuda_runtime.h>

#include <optional>
#include <vector>

#include "../cuda/launch.hpp"
#include "device.hpp"
#include "setup.hpp"

namespace spkb {

// A film/print set-up pair with its device tables, built once per pipeline.
struct DeviceTables {
    DevBuffer table;              // L x L spectral table, float4 texels (R, G, B, 0)
    DevBuffer patches;            // the same as (L - 1)^2 patches of 4 x 4 RGB texels (kPatchFloats each)
    DevBuffer curves;             // x[K] | inv[K] | y[3K] | y0[3K] (the DIR couplers' pre-inverted curve)
    DevBuffer gaxis, ginv, glayers;
    DevBuffer paper;              // x[K] | r[K] | y[K][3]
    DevBuffer cmax;               // 64 x 720
    DevBuffer edr;                // the EDR tone map's target_log2_y (binary32), when EDR is on
};

struct Pipeline {
    std::shared_ptr<const FilmSetup> film;
    std::shared_ptr<const PrintSetup> print;
    DeviceTables dev;
};

struct RenderCtx;
// Whether the back-reflection halation's highlight headroom runs (reference src/fx/halation.cpp:64-66).
bool headroom_applies(const HalationParams& h);
// The print glare's field for a w x h print (reference src/fx/glare.cpp:27-50): one lognormal value per
// pixel (mean percent amount, sd roughness percent amount, stream 200, ctx.print_seed) on all channels,
// blurred by 0.5 px x rho_tier x sqrt(amount); empty when the glare draws nothing or the negative is
// scanned directly.
Plane glare_plane(RenderCtx& ctx, const Pipeline& p, uint32_t w, uint32_t h);

// Upload a pipeline's tables (stream-ordered, then synchronised).
void upload_tables(Pool& pool, cudaStream_t s, Pipeline& p);

// Receives the render's progress nodes: one call per stage of the reference's pipeline, with its label
// (reference src/core/render.hpp:52-84), before the stage's work is enqueued. The session's record checks
// its cancel flag there and throws SPK_ERR_CANCELLED.
class ProgressSink {
public:
    virtual void node(const char* label) = 0;

protected:
    ~ProgressSink() = default;
};

// The node() calls a develop and a print make (reference src/film/develop.cpp:64-78,
// src/print/run.cpp:89-99): the totals behind the progress percentage.
uint32_t film_node_count(const FilmSetup& f);
uint32_t print_node_count(const PrintSetup& s);

struct RenderCtx {
    Pool& pool;
    cudaStream_t stream;
    ProgressSink* progress = nullptr;  // null: no progress, not cancellable (warm-up, adjoint, hooks)
    void node(const char* label) const {
        if (progress) progress->node(label);
    }
    double pitch_um = 0.0;
    double rho_tier = 1.0;
    std::optional<double> ae_ev = std::nullopt;
    uint32_t print_seed = 0;  // the print glare's seed (0 when the glare draws nothing)  // the auto-exposure meter's EV for the develop (none: no scale)
    // optional per-stage timing: events recorded around each stage when set
    struct Timer* timer = nullptr;
    // the print stage: -1 the binary32 print kernel, else a SpectralMode of the spectral-mode kernel at
    // print_bins wavelengths (81, or 401 resampled to 1 nm); contraction_out (device, may be null) then
    // receives the enlarger integral of every pixel (3 floats)
    int print_mode = -1;
    uint32_t print_bins = SPKB_NL;
    float* contraction_out = nullptr;
    // the print side's copy to the output image's host pixels, in row bands on copy_stream (events from
    // band_events, grown as needed), overlapping the next band's kernels; null: no banded copy
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t>* band_events = nullptr;
};

// Stage timing with CUDA events on the render stream (bench and profile entry points).
struct Timer : dev::LaunchHook {
    struct Mark {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<Mark> marks;    // stages
    std::vector<Mark> kernels;  // every kernel launch inside them
    void begin(const char* name, cudaStream_t s);
    void end(cudaStream_t s);
    void before(const char* kernel, cudaStream_t s) override;
    void after(cudaStream_t s) override;
    void reset();
    ~Timer() override;
};

// film side: raw source plane -> developed negative density plane (a fresh persistent plane)
// counts_out: nullptr, or device memory for 9 floats per pixel receiving the grain's Poisson counts;
// lam_out: nullptr, or the same for the draws' lambdas (sub-layer grain)
Plane develop(RenderCtx& ctx, const Pipeline& p, const Plane& source, uint32_t film_seed,
              const std::optional<HalationOverride>& hov, float* counts_out = nullptr, float* lam_out = nullptr);

// The spectral-mode kernel's tables of a print set-up at the live print run, at 81 or 401 wavelengths.
void spectral_tables_n(const PrintSetup& s, const PrintRun& r, uint32_t bins, SpectralTablesN& out);

// The print kernel's arguments for a negative of `pixels` pixels at the live parameters.
PrintArgs print_args(const Pipeline& p, const LiveParams& live, uint32_t pixels);
// The fused scanner kernel's arguments for a w x h frame written with row pitch stride_px; false when the
// frame or the scanner's blurs need the separate passes (a recursive blur, a frame narrower than the halo).
bool scan_args(const Pipeline& p, double rho_tier, uint32_t w, uint32_t h, uint32_t stride_px, ScanArgs& out);

// print side: negative -> RGBA16 into img->dev (row pitch img->stride_px). With to_host and a copy stream
// in ctx, the rows are also copied to img->host, band by band as they are written, and true is returned
// (the stream then orders after the copies); false: no host copy was made.
bool print_scan_encode(RenderCtx& ctx, const Pipeline& p, const LiveParams& live, const Plane& negative,
                       OutputImage* img, bool to_host = false);
// The print side's progress nodes for a print that runs as one fused launch chain (the batch plans):
// every label of print_node_count, in order.
void print_nodes(RenderCtx& ctx, const PrintSetup& s);

// The adjoint of the render. The differentiated output y is the scanned linear RGB (print, scanner lens
// blur and unsharp mask; before the output transfer function and the 16-bit encode) of the source frame,
// developed with the grain counts of film_seed held fixed. Device pointers, 3 floats per pixel:
//   y_out (may be null)  receives y;
//   g_y (null: y only)   the gradient of a loss with respect to y;
//   g_x                  receives the gradient with respect to the source frame.
// grad_params (host, n_params entries, may be null) receives the gradient with respect to
//   [print_exposure, m_filter_shift, y_filter_shift, halation weight 0..K-1, halation sigma 0..K-1,
//    density-curve parameter (layer c, node j) at 3 + 2K + 16 c + j],
// K the components of the halation override (none without one). A weight's or sigma's gradient is along
// a common change of its three channels; the curve parameters are the hat functions of vjp.hpp.
void render_vjp(RenderCtx& ctx, const Pipeline& p, const LiveParams& live, const Plane& source, uint32_t film_seed,
                const std::optional<HalationOverride>& hov, float* y_out, const float* g_y, float* g_x,
                double* grad_params, uint32_t n_params);

// The DIR-coupler diffusion (reference src/fx/dir_blur.hpp:15-19, dir_blur.cpp:14-38) at a pixel pitch: a
// core Gaussian of 20 um with weight 1 - 0.06 and the exponential surrogate of a 200 um tail with weight 0.06.
std::vector<MixtureComponent> dir_diffusion_components(double pitch_um);

// The blur machinery on device planes (exposed for the tests' stage entry points).
void gaussian(RenderCtx& ctx, const Plane& in, const Plane& dst, const Vec3& sigma);
void gaussian_mixture(RenderCtx& ctx, const Plane& in, const Plane& out, const std::vector<MixtureComponent>& comps);

// Checks that a parameter set stays inside this build's render path; SPK_ERR_USER with the reason.
void check_supported(const ParamSet& p);

}  // namespace spkb
