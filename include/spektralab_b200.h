/* spektralab B200 extensions: entry points with no counterpart in the reference engine's C ABI.
 *
 * Conventions are those of spektralab.h: C linkage, no exceptions cross, a negative spk_status and a
 * message in spk_last_error on failure. Host pointers unless stated.
 */
#ifndef SPEKTRALAB_B200_H
#define SPEKTRALAB_B200_H

#include "spektralab.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- test and benchmark configuration ----
 *
 * spkx_session_set_halation(session, n, weights, sigmas_px, strength)
 *   replace the session's halation with a Gaussian mixture given in pixels:
 *     H(x) = sum_k weight[k][c] G_{sigma[k][c]}(x);  raw := raw / (1 + A_c) + A_c H(raw) / (1 + A_c)
 *   weights and sigmas_px hold n x 3 doubles, strength 3; n = 0 restores the film's own halation
 *   (its preset through the scatter and bounce models). The scatter stage is dropped while set.
 *   drops every cached negative. SPK_ERR_INVALID_ARG for n > 8 or a NULL array with n > 0.
 *   The halation configurations of the benchmark workloads (two components of given sigma in pixels)
 *   cannot be expressed through the reference's parameters, so tests and bench set them here, and
 *   set the same mixture on the reference oracle.
 */
SPK_API spk_status spkx_session_set_halation(spk_session* session, uint32_t n, const double* weights,
                                             const double* sigmas_px, const double* strength);

/* spkx_session_profile(session, tier, reprint, steps, out_json)
 *   render (reprint = 0) or reprint (reprint = 1) `steps` times on the device, with no host copy of the
 *   result, and report per-stage device times from CUDA events on the session's stream:
 *     {"steps": K, "total_ms": [..K], "stages": {"expose": [...], ...}, "pixels": P}
 *   before every step the L2 cache is flushed by writing a 256 MiB buffer (untimed).
 *   a render step develops afresh each time; a reprint step prints the cached negative.
 */
SPK_API spk_status spkx_session_profile(spk_session* session, const char* tier, int32_t reprint, uint32_t steps,
                                        char** out_json);

/* spkx_session_negative(session, tier, out, capacity_floats)
 *   copy the tier's cached negative (3 floats per pixel) to host memory; SPK_ERR_USER when none is cached.
 */
SPK_API spk_status spkx_session_negative(spk_session* session, const char* tier, float* out, size_t capacity_floats);

/* spkx_session_meter(session, out_json)
 *   the auto-exposure meter's seven EV values (center_weighted, average, median, balanced, center,
 *   protect_highlights, protect_shadows) as a JSON object; meters the frame first when no meter is kept.
 *   SPK_ERR_USER when auto_exposure is off.
 */
SPK_API spk_status spkx_session_meter(spk_session* session, char** out_json);

/* spkx_session_tier_image(session, tier, out, capacity_floats, width, height)
 *   the tier's image (the frame downscaled to the tier's long edge, made on first use and kept; the frame
 *   itself when it fits): its size in *width, *height and, when out is not NULL and capacity_floats
 *   holds 3 floats per pixel, its pixels.
 */
SPK_API spk_status spkx_session_tier_image(spk_session* session, const char* tier, float* out, size_t capacity_floats,
                                          uint32_t* width, uint32_t* height);

/* spkx_session_develop_debug(session, tier, film_seed, negative, counts)
 *   develop the tier's frame once more with the given film seed, without touching the cache:
 *   negative receives 3 floats per pixel, counts (may be NULL) the grain's Poisson counts, 9 floats per
 *   pixel [channel][sub-layer]. The first render of a session uses the seed sequence's first draw,
 *   0x4abea221, so this reproduces its negative and tells which counts it drew.
 */
SPK_API spk_status spkx_session_develop_debug(spk_session* session, const char* tier, uint32_t film_seed,
                                              float* negative, float* counts);

/* spkx_session_develop_draws(session, tier, film_seed, counts, lambdas)
 *   the grain's draws of a develop with the given film seed (sub-layer grain): counts and lambdas receive
 *   9 floats per pixel each, [c][l], the Poisson count and the lambda it was drawn with. Draw (c, l) of
 *   pixel y * width + x uses the sampler's stream c + 10 l, so spkx_sampler_poisson over one (c, l)
 *   plane of lambdas, with that stream and seed, reproduces the counts.
 */
SPK_API spk_status spkx_session_develop_draws(spk_session* session, const char* tier, uint32_t film_seed, float* counts,
                                             float* lambdas);

/* spkx_session_setup_json(session, out_json)
 *   the narrowed kernel constants of the session's pipeline, for set-up parity checks:
 *   input matrix, curve tables, grain tables and constants at a given pitch, enlarger and scan
 *   tables of the current live parameters, paper curve, CAM16 arguments and the C_max table.
 */
SPK_API spk_status spkx_session_setup_json(spk_session* session, double pitch_um, char** out_json);

/* spkx_setup_json(resources_dir, params_delta_json, pitch_um, out_json)
 *   the same constants for the parameters an spk_open with this delta would use, built on the host
 *   alone (no device, no engine): the binary64 set-up can be checked on a machine without a GPU.
 */
SPK_API spk_status spkx_setup_json(const char* resources_dir, const char* params_delta_json, double pitch_um,
                                   char** out_json);

/* ---- stage-level test entry points (host arrays in and out; run on the current device) ---- */

/* Poisson counts (as floats) of the grain sampler for pixel index i = 0..n-1 on one stream and seed */
SPK_API spk_status spkx_sampler_poisson(const float* lam, float* counts, uint32_t n, uint32_t stream,
                                        uint32_t seed);
/* the Box-Muller lognormal value for pixel index i = 0..n-1 */
SPK_API spk_status spkx_sampler_lognormal(float* out, uint32_t n, float mean, float stddev, uint32_t stream,
                                          uint32_t seed);
/* Philox4x32-10 of n (counter[4], key[2]) pairs into out[4n] */
SPK_API spk_status spkx_philox(const uint32_t* counters, const uint32_t* keys, uint32_t* out, uint32_t n);

/* Test hook of the failure path (no counterpart in the reference engine): the SM clocks a stage wait of
 * the tensor-core print kernel may take before it gives up (0: the normal limit, about 2 s). With a limit
 * of a few clocks a wait runs out at once; the kernel then stops issuing work, drains the MMAs it issued
 * under the normal limit, frees its tensor memory and flags the failure, and the render returns
 * SPK_ERR_GPU with the context still usable. Process-wide; set it back to 0 afterwards. */
SPK_API spk_status spkx_test_set_tc_wait_limit(int64_t cycles);

/* Test hooks of the recursive blur's column pass (no counterpart in the reference engine), which loads its
 * strips by TMA and waits on an mbarrier. spkx_test_set_iir_wait_limit: the SM clocks a strip wait may
 * take before it gives up (0: the normal limit, about 2 s; process-wide, set it back to 0 afterwards). A
 * wait that gives up is counted, then waits again under the normal limit for the copies in flight, and
 * the blur's result is unchanged. spkx_test_take_iir_waits_given_up: the count since the last call, reset
 * to 0. */
SPK_API spk_status spkx_test_set_iir_wait_limit(int64_t cycles);
SPK_API spk_status spkx_test_take_iir_waits_given_up(uint32_t* count);

/* the Gaussian blur of a w x h RGB float plane (3 floats per pixel) with per-channel sigma in pixels,
 * by the engine's FIR / recursive branch rule */
SPK_API spk_status spkx_gaussian(const float* in, float* out, uint32_t w, uint32_t h, const double* sigma3);

/* ---- batched renders (no counterpart in the reference engine) ----
 *
 * spkx_render_batch(sessions, n, tier, reprint, results, out_json)
 *   spk_render (reprint = 0) or spk_reprint (reprint != 0) of n distinct sessions of one engine in one call;
 *   results[i] is what that call would give sessions[i], pixel for pixel, and is released with
 *   spk_result_free. The film side of each frame runs on its session's stream; the print side of the frames
 *   runs as one CUDA graph: per-frame launches spread over worker streams, or one persistent print launch and
 *   one persistent scanner launch for every frame. The first batch of a list of frame sizes times each plan
 *   on the device and keeps the fastest for that list. results[i].elapsed_ms is the time from the start of
 *   the call's device work to that frame's result in host memory. out_json (may be NULL) receives
 *   {"plan": ..., "tuning_ms": ..., "frame_done_ms": [...]}, with "candidates_ms" (each plan's device time)
 *   after a timed choice. On failure every result is zeroed.
 *   SPK_ERR_INVALID_ARG: NULL arrays, n = 0, a session twice, sessions of different engines, unknown tier.
 */
SPK_API spk_status spkx_render_batch(spk_session* const* sessions, uint32_t n, const char* tier, int32_t reprint,
                                     spk_result* results, char** out_json);

/* spkx_engine_batch_plan(engine, plan)
 *   pins the plan of every later spkx_render_batch of this engine ("frames:K", K 1..16: per-frame launches on
 *   K worker streams; "persistent:S:C": items of S pixels, S even, over C CTAs; "persistent:S:C:G": the
 *   same in G consecutive groups of frames, G 1..1024, each group's result copies overlapping the next
 *   group's launches); NULL or "" restores the timed choice. SPK_ERR_INVALID_ARG for any other string.
 */
SPK_API spk_status spkx_engine_batch_plan(spk_engine* engine, const char* plan);

/* ---- the print's spectral integrals on the tensor cores (no counterpart in the reference engine) ----
 *
 * spkx_session_set_print_mode(session, mode, bins)
 *   selects the arithmetic of the print's two spectral integrals (enlarger and scan, reference
 *   kernels/print.metal:165-189) for the session's later renders, reprints and spkx_print_negative calls:
 *     "fp32"          the binary32 print kernel (the default; at 401 wavelengths the spectral-mode kernel's
 *                     binary32 path, which performs the same operations)
 *     "fp32_generic"  the spectral-mode kernel's binary32 path (at 81 wavelengths equal to "fp32" bit for bit)
 *     "fp64"          both integrals in binary64 from the binary64 set-up tables
 *     "tf32", "bf16"  the sums over wavelengths on the tensor cores (tcgen05), binary32 accumulation
 *     "bf16x3"        the same with BF16 hi + lo splits of both operands (all four products)
 *   bins: 81 (the resources' 5 nm grid) or 401 (1 nm, the binary64 tables interpolated linearly).
 *   The stages around the integrals stay binary32. SPK_ERR_INVALID_ARG for another mode or bins.
 *
 * spkx_print_negative(session, negative, width, height, rgba16, row_stride_px, contraction, print_ms)
 *   the print side of a render (print, scanner, output encode) of a given negative with the session's
 *   parameters and print mode. negative: device memory, width x height x 3 floats (dye densities);
 *   rgba16: device memory, row pitch row_stride_px pixels; contraction (device, may be NULL; spectral-mode
 *   kernels only) receives the enlarger integral R_k of every pixel (3 floats); print_ms (host, may be
 *   NULL) receives the device time of the print kernel. Synchronous on the session's stream.
 */
SPK_API spk_status spkx_session_set_print_mode(spk_session* session, const char* mode, uint32_t bins);
SPK_API spk_status spkx_print_negative(spk_session* session, const float* negative, uint32_t width, uint32_t height,
                                       uint16_t* rgba16, uint32_t row_stride_px, float* contraction, double* print_ms);

/* ---- the render's adjoint (no counterpart in the reference engine) ----
 *
 * spk_render_vjp(session, tier, film_seed, grad_output, grad_input, grad_params, n_params, output)
 *   The differentiated output is the scanned linear RGB of the session's frame: the render up to the
 *   scanner's lens blur and unsharp mask, before the output transfer function and the 16-bit encode, with
 *   the grain held as fixed noise (the Poisson counts of film_seed). Host arrays of 3 floats per pixel:
 *     output       (may be NULL) receives that linear RGB;
 *     grad_output  (NULL: the output alone is computed) the gradient of a loss with respect to it;
 *     grad_input   receives the gradient with respect to the session's source frame (RGB).
 *   grad_params (n_params doubles) receives the gradient with respect to
 *     [print_exposure, m_filter_shift, y_filter_shift, halation weight 0..K-1, halation sigma 0..K-1,
 *      density-curve parameter theta[c][j] for film layer c = 0..2 and node j = 0..15 at 3 + 2K + 16c + j],
 *   K the components set by spkx_session_set_halation (none otherwise; entries past the list are 0). A
 *   halation weight or sigma is taken as one value for the three channels. theta[c][j] adds
 *   theta phi_j(k) to entry k of layer c's K-entry density-curve table, phi_j(k) = max(0, 1 - |15k/(K-1) - j|)
 *   (16 hat functions over the table; the curve's lookup interpolates the perturbed entries linearly).
 *   Blur passes are recomputed, not stored; the recursive blurs run transposed. Refused with
 *   SPK_ERR_UNSUPPORTED: grain below full strength or without sub-layers, halation components whose
 *   three channels differ in sigma.
 */
SPK_API spk_status spk_render_vjp(spk_session* session, const char* tier, uint32_t film_seed, const float* grad_output,
                                  float* grad_input, double* grad_params, uint32_t n_params, float* output);

/* ---- allocation-free entry point (no counterpart in the reference engine) ----
 *
 * spkx_gaussian_noalloc(in, out, w, h, sigma3, stream)
 *   The Gaussian blur of spkx_gaussian for callers that cannot have device memory allocated on their
 *   behalf: a host application that owns all device memory through its own allocator and calls its
 *   plug-ins inside a per-frame render callback, or a real-time pipeline in which cudaMalloc's latency and
 *   implicit synchronisation are not allowed. The caller passes device buffers (w x h x 3 floats each;
 *   out may equal in) and a cudaStream_t (NULL: the legacy default stream); the work is enqueued on that
 *   stream and the call returns without waiting. It allocates nothing: the intermediate planes live in a
 *   fixed 16 MiB array compiled into the library, so w * h must not exceed 699,050 pixels (2^21 floats
 *   per plane); larger frames are refused with SPK_ERR_INVALID_ARG. Every GPU that loads the library
 *   keeps the array until the process exits. The first call in each CUDA context (the device's primary
 *   context, or a driver context the host made current) looks up the array's address in that context and
 *   keeps it for later calls in the same context (keyed by the driver's context id, so a new context or a
 *   reset device gets a fresh lookup); make that first call before any stream capture. All calls in a
 *   context share the one array and leave their data in it, so calls whose work overlaps on the GPU race:
 *   order them on one stream, or wait for one before starting the next on another. Buffers that start on
 *   16-byte boundaries (as cudaMalloc's do) let the recursive channels (sigma >= 3) run the block-parallel
 *   kernels; other buffers take slower one-thread-per-line kernels (the same recurrence, rounded in a
 *   different order: results agree within the blur's tolerances).
 */
SPK_API spk_status spkx_gaussian_noalloc(const float* in, float* out, uint32_t w, uint32_t h, const double* sigma3,
                                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SPEKTRALAB_B200_H */
