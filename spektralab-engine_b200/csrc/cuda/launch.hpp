// Host-callable launchers of the sm_100a render kernels. Planes are interleaved binary32 RGB
// (12 bytes per pixel, row-major, top row first) in device memory; every launcher enqueues on the
// given stream and returns without synchronising.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"

namespace spkb::dev {

// Observation of kernel launches: every launcher below counts itself, and when the calling thread has
// a hook set, brackets its launch with before/after (the hook records CUDA events on the stream).
struct LaunchHook {
    virtual void before(const char* kernel, cudaStream_t s) = 0;
    virtual void after(cudaStream_t s) = 0;
    virtual ~LaunchHook() = default;
};
void set_launch_hook(LaunchHook* hook);  // per thread; nullptr clears
uint64_t launch_count();                 // kernels launched by this library since load

// Brackets one launch: counts it and calls the thread's hook.
struct Probe {
    cudaStream_t s;
    Probe(const char* kernel, cudaStream_t stream);
    ~Probe();
};

// Raises a kernel's dynamic shared-memory limit to `bytes` in the current context, once (a later call in
// the same context asking no more is a no-op), so that launches inside a stream capture make no attribute
// call. A new context (a host's own driver context, or one after a device reset) sets it afresh.
void ensure_smem(const void* kernel, int bytes);

// The driver's unique id of the current CUDA context; 0 when none is current or the driver cannot say.
unsigned long long current_context_id();

// Tier downscale: the vertical prefilter src -> dst (same size), then the horizontal prefilter at the
// bilinear sample points fused with the blend, v (in_w x in_h) -> dst (out_w x out_h).
void tier_blur_v(const float* src, float* dst, const TierBlurArgs& a, cudaStream_t s);
void tier_resample(const float* v, float* dst, const TierResampleArgs& a, cudaStream_t s);
// Input transfer decode and geometry: src (src_w x src_h) -> dst (dst_w x dst_h).
void prepare(const float* src, float* dst, const PrepareArgs& a, cudaStream_t s);

// The auto-exposure meter's statistics of the meter image into *a.out (13 doubles); a.sel must hold the
// six ranks with zero prefixes, masks and histograms. a.partial holds meter_partial_doubles() doubles.
size_t meter_partial_doubles();
void meter_stats(const MeterArgs& a, cudaStream_t s);

// The frame maximum of n floats (NaN skipped) as an order-preserving integer in *out_ordered, and as a
// float (plane_max_value); the back-reflection headroom (reading the clip from device memory) and the
// highlight boost.
void plane_max(const float* p, size_t n, uint32_t* out_ordered, cudaStream_t s);
void plane_max_value(const uint32_t* ordered_max, float* out, cudaStream_t s);
void headroom(float* p, uint32_t pixels, const uint32_t* clip_ordered, float headroom_ev, cudaStream_t s);
void boost(float* p, size_t n, float x0, float r, float a, float k, cudaStream_t s);

// RGB -> film exposure H (Mitchell bicubic of the spectral table, L x L float4 texels), times the
// compensation gain.
// patches (may be null): the table as 4 x 4 patches (kPatchFloats floats per base pair, (L - 1)^2 pairs),
// read by the vectorised kernel when both planes are 16-byte aligned; else the texel kernel reads table4.
void expose(const float* rgb, float* h, const float* table4, const float* patches, const ExposeArgs& a,
            cudaStream_t s);

// Separable FIR: vertical pass in -> out (no accumulation).
void fir_v(const float* in, float* out, uint32_t w, uint32_t h, const FirTaps& t, cudaStream_t s);
// Horizontal pass with the accumulation of the last pass (ACC_NONE / ZERO / PLANE with weights).
void fir_h(const float* in, float* out, const float* acc, uint32_t w, uint32_t h, const FirTaps& t, int mode,
           const float weight[3], cudaStream_t s);
// Recursive Gaussian, horizontal: in -> out (forward then backward along each row).
void iir_h(const float* in, float* out, uint32_t w, uint32_t h, const IirCoefs& c, cudaStream_t s);
// Recursive Gaussian, vertical: work holds the horizontal result and is overwritten with the forward
// pass; out := y, 0 + w y or acc + w y.
void iir_v(float* work, float* out, const float* acc, uint32_t w, uint32_t h, const IirCoefs& c, int mode,
           const float weight[3], cudaStream_t s);
// The recursive Gaussian of one direction with its tangent along sigma (the adjoint's sigma gradient):
// (in, in_dot) -> (out, out_dot), dc the coefficients' derivatives; work planes hold the forward pass.
void iir_tangent(const float* in, const float* in_dot, float* work, float* work_dot, float* out, float* out_dot,
                 uint32_t w, uint32_t h, bool vertical, const IirCoefs& c, const IirCoefs& dc, cudaStream_t s);
// out = a x + b y per channel (y reads as 0 when y == nullptr).
void lincomb(const float* x, const float* y, float* out, size_t pixels, const float a[3], const float b[3],
             cudaStream_t s);
void copy(const float* x, float* out, size_t pixels, cudaStream_t s);

// DIR couplers: exposure -> the coupler correction chi (before its diffusion blur).
void coupler_source(const float* exposure, float* chi, const CouplerArgs& a, cudaStream_t s);

// log10 exposure -> density curves -> grain draw (grain mode) or density (no grain).
void develop(const float* exposure, float* out, const DevelopArgs& a, uint32_t w, uint32_t h, cudaStream_t s);
// The grain's log(k!) table on the current device (once per process; waits for it on s). The engine calls
// it at creation; develop calls it too, before its first grain launch on a device.
void develop_prepare(cudaStream_t s);

// negative density -> linear output RGB (enlarger, gain, paper, scan, XYZ -> RGB, CAM16 gamut).
void print(const float* neg, float* rgb, const PrintArgs& a, cudaStream_t s);

// The print stage with the spectral integrals in the given SpectralMode (print_tc.cu): host_tab the
// tables on the host (their binary32 part goes into the kernel's parameters), tab the same in device
// memory; host_tab.nl_pad must be 96 or SPKB_NL_MAX. contraction (may be null) receives the enlarger
// integral R_k of every pixel (3 floats). *err (device) is or-ed with 1 when a tensor-core wait gave up.
void print_spectral(const PrintArgs& a, const SpectralTablesN& host_tab, const SpectralTablesN* tab, int mode,
                    const float* neg, float* rgb, uint32_t n, float* contraction, uint32_t* err, cudaStream_t s);
bool print_spectral_supported(uint32_t nl_pad);
// The limit of the spectral-mode kernel's stage waits in SM clocks (0: the normal limit); a test hook.
void set_tc_wait_limit(long long cycles);

// The print-preview table render: negative densities -> trilinear table -> RGBA16 (row pitch a.stride).
void print_lut(const float* neg, uint16_t* out, const PrintLutArgs& a, cudaStream_t s);

// The print glare's lognormal field: one value per pixel (stream 200, the print seed) on three channels.
void glare_field(float* out, uint32_t pixels, float mean, float sd, uint32_t seed, cudaStream_t s);

// (optional unsharp combine with g) -> transfer function -> RGBA16 with row pitch e.stride.
void encode(const float* rgb, const float* g, uint16_t* out, uint32_t w, uint32_t h, const EncodeArgs& e,
            cudaStream_t s);

// The scanner stage in one tiled pass: lens blur (radius a.r1), unsharp (a.r2, when a.e.unsharp), matrix,
// transfer function, RGBA16. scan_encode_fits tells whether the tiled kernel takes this frame and these radii.
bool scan_encode_fits(uint32_t w, uint32_t h, int r1, int r2);
void scan_encode(const float* rgb, uint16_t* out, uint32_t w, uint32_t h, const ScanArgs& a, cudaStream_t s);
// the same for output rows row0 .. row1 - 1 only (row0 a multiple of scan_tile_rows(); the rows' halo of
// the print output must be written)
void scan_encode_rows(const float* rgb, uint16_t* out, uint32_t w, uint32_t h, uint32_t row0, uint32_t row1,
                      const ScanArgs& a, cudaStream_t s);
constexpr uint32_t scan_tile_rows() { return 32; }

// A separable FIR (taps[0..2r], the same for the three channels) with both passes in one tiled kernel;
// out must not alias in. fir_tile_fits tells whether the tiled kernel takes this frame and radius.
bool fir_tile_fits(uint32_t w, uint32_t h, int r);
void fir_tile(const float* in, float* out, uint32_t w, uint32_t h, int r, const float* taps, cudaStream_t s);

// The print and scanner stages of many frames, each in one persistent launch of `ctas` CTAs: print over
// items of item_px pixels (item_frame / item_first per item, ordered by frame; frames in device memory),
// the scanner over the frames' concatenated 32 x 32 tile lists (frames in device memory, ordered by
// first_tile; r1, r2 the radii every frame shares, or -1 for frames that differ).
// enl and scan (host, may be null): spectral tables every frame shares, which the kernel then takes in its
// parameters (the constant bank) instead of staging them per frame in shared memory.
void print_batch(const BatchPrintFrame* frames, const uint32_t* item_frame, const uint32_t* item_first,
                 uint32_t n_items, uint32_t item_px, uint32_t ctas, const SpectralPairs* enl,
                 const SpectralPairs* scan, cudaStream_t s);
void scan_encode_batch(const BatchScanFrame* frames, uint32_t n_frames, uint32_t n_tiles, int r1, int r2,
                       uint32_t ctas, cudaStream_t s);
// Sets the scanner kernels' shared-memory limits on the current device (before a stream capture).
void scan_prepare();
uint32_t scan_tiles(uint32_t w, uint32_t h);  // 32 x 32 tiles of a w x h frame
uint32_t scan_tiles_x(uint32_t w);

// host frame (channels 3 or 4, already on the device) -> interleaved RGB plane, non-finite -> 0
void source_copy(const float* raw, float* out, size_t pixels, uint32_t channels, cudaStream_t s);
// write `bytes` (a multiple of 16) with a constant word (the L2 flush between timed steps)
void fill(void* p, size_t bytes, uint32_t v, cudaStream_t s);

// Test entry points: the sampler over an array of lambdas (counts as floats) and raw Philox blocks.
void sampler_poisson(const float* lam, float* out, uint32_t n, uint32_t stream, uint32_t seed, cudaStream_t s);
void sampler_lognormal(float* out, uint32_t n, float mean, float stddev, uint32_t stream, uint32_t seed,
                       cudaStream_t s);
void philox_blocks(const uint32_t* ctr, const uint32_t* key, uint32_t* out, uint32_t n, cudaStream_t s);

}  // namespace spkb::dev
