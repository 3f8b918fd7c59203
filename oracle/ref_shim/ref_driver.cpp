// Test infrastructure (oracle): stage-level entry points over the reference engine's own code, built
// into oracle/_ref/libspektralab_ref.so beside its spk_* ABI. Everything here calls the reference's
// functions (src/film, src/print, src/fx, src/session); the only steps restated are the session's
// open sequence (src/session/session.cpp:121-197) and the film-side stage order of
// src/film/develop.cpp:101-236, so that a halation mixture given in pixels can be put in place of
// the preset (the benchmark workloads name their halation that way; no schema field reaches it).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "film/film_internal.hpp"
#include "film_shared.h"
#include "fx/dir_blur.hpp"
#include "fx/fx_internal.hpp"
#include "fx/grain.hpp"
#include "fx/halation.hpp"
#include "fx/rng.hpp"
#include "params/params.hpp"
#include "print/internal.hpp"
#include "print/print.hpp"
#include "session/engine.hpp"
#include "session/tiers.hpp"
#include "spektralab.h"
#include "util/error.hpp"
#include "util/json.hpp"
#include "util/numeric.hpp"

using namespace spk;

namespace {

struct Built {
    std::shared_ptr<const film::FilmSetup> film;
    std::shared_ptr<const print::PrintSetup> print;
    std::unique_ptr<params::ParamSet> p;
    bool product_defaults = false;
};

Built build(Engine& e, const char* delta_text) {
    params::Delta d = params::validate_delta(e.schema(), delta_text ? delta_text : "", params::DeltaContext::Open);
    Built b;
    b.product_defaults = d.product_defaults.value_or(false);
    b.p = std::make_unique<params::ParamSet>(e.schema_ptr());
    params::ParamSet& p = *b.p;
    for (const auto& [fid, v] : d.fields)
        if (fid == params::id(params::P::film_stock) || fid == params::id(params::P::print_stock)) p.set(fid, v);
    const res::Resources& res = e.resources();
    auto film = res.profile(p.s(params::P::film_stock));
    auto paper = res.profile(p.s(params::P::print_stock));
    auto digest = [&] {
        if (auto pack = res.filters.lookup_with_alias(p.s(params::P::print_stock), p.s(params::P::enlarger_illuminant),
                                                      film->id, film->base_id)) {
            p.set(params::P::c_filter_neutral, (*pack)[0]);
            p.set(params::P::m_filter_neutral, (*pack)[1]);
            p.set(params::P::y_filter_neutral, (*pack)[2]);
        }
    };
    digest();
    p.set(params::P::output_color_space, "ProPhoto RGB");
    p.set(params::P::output_cctf_encoding, true);
    params::apply_delta(p, d);
    digest();
    b.film = film::build_film_setup({p, film, res, e.gpu(), e.device()});
    b.print = print::build_print_setup({p, *b.film, paper, res, e.gpu(), &e.cam16_cache(), e.device(), !b.product_defaults});
    return b;
}

// develop() with the bounce mixture replaced (stage order of src/film/develop.cpp:101-236 for the
// identity geometry, no auto exposure, no boost and no headroom)
gpu::Plane develop_override(core::RenderContext& ctx, const film::FilmSetup& setup, const gpu::Plane& src,
                            uint32_t seed, uint32_t n, const double* weights, const double* sigmas,
                            const double* strength) {
    const film::FilmSetup::Impl& s = setup.impl();
    const params::ParamSet& b = s.params;
    using params::P;
    gpu::Plane plane = ctx.scratch(src.w, src.h);
    {
        SpkFilmUpsampleArgs a{};
        a.n = uint32_t(src.pixels());
        a.L = s.table->size;
        for (size_t i = 0; i < 9; ++i) a.a[i] = s.input_matrix_f32[i];
        gpu::Batch bt = ctx.gpu.batch();
        bt.dispatch_1d(ctx.kernel("spk_film_upsample"), a.n,
                       {gpu::Arg::plane(src), gpu::Arg::plane(plane), gpu::Arg::buffer(s.table->f32), gpu::Arg::value(a)});
        bt.commit_and_wait();
    }
    {
        const float g = num::f32(std::pow(2.0, b.f(P::exposure_compensation_ev)));
        if (g != 1.0f) film::run_scale(ctx, plane, g);
    }
    if (b.f(P::lens_blur_um) > 0.0) fx::lens_blur(ctx, plane, b.f(P::lens_blur_um));
    if (n > 0) {
        std::vector<fx::MixtureComponent> comps(n);
        for (uint32_t k = 0; k < n; ++k)
            for (int c = 0; c < 3; ++c) {
                comps[k].weight[size_t(c)] = weights[3 * k + c];
                comps[k].sigma[size_t(c)] = sigmas[3 * k + c];
            }
        fx::Vec3 ma{}, mb{};
        for (int c = 0; c < 3; ++c) {
            ma[size_t(c)] = 1.0 / (1.0 + strength[c]);
            mb[size_t(c)] = strength[c] / (1.0 + strength[c]);
        }
        gpu::Batch bt = ctx.gpu.batch();
        gpu::Plane H = ctx.scratch(src.w, src.h);
        fx::detail::encode_mixture(ctx, bt, plane, H, comps);
        fx::detail::encode_lincomb(ctx, bt, ma, plane, mb, &H, plane);
        bt.commit_and_wait();
    } else if (s.halation.active) {
        fx::halation(ctx, plane, s.halation);
    }
    {
        SpkFilmLogArgs a{uint32_t(plane.floats())};
        gpu::Batch bt = ctx.gpu.batch();
        bt.dispatch_1d(ctx.kernel("spk_film_log"), a.n, {gpu::Arg::plane(plane), gpu::Arg::value(a)});
        bt.commit_and_wait();
    }
    // the curves develop into a second plane when the couplers need the log exposure again
    gpu::Plane developed = s.couplers ? ctx.scratch(plane.w, plane.h) : plane;
    {
        SpkFilmCurvesArgs a{uint32_t(plane.pixels()), s.curves.K, 0u};
        gpu::Batch bt = ctx.gpu.batch();
        bt.dispatch_1d(ctx.kernel("spk_film_curves"), a.n,
                       {gpu::Arg::plane(plane), gpu::Arg::plane(developed), gpu::Arg::buffer(s.curve_buffer),
                        gpu::Arg::value(a)});
        bt.commit_and_wait();
    }
    if (s.couplers) {
        // DIR couplers (src/film/develop.cpp:203-226): the first development becomes the inhibitor source,
        // is diffused, and corrects the log exposure before the second lookup through the curves
        SpkFilmCouplerArgs ca{};
        ca.n = uint32_t(developed.pixels());
        ca.positive = s.positive ? 1u : 0u;
        for (size_t i = 0; i < 9; ++i) ca.m[i] = s.coupler_m_f32[i];
        for (size_t c = 0; c < 3; ++c) ca.dmax[c] = s.dmax_f32[c];
        {
            gpu::Batch bt = ctx.gpu.batch();
            bt.dispatch_1d(ctx.kernel("spk_film_coupler_source"), ca.n,
                           {gpu::Arg::plane(developed), gpu::Arg::value(ca)});
            bt.commit_and_wait();
        }
        fx::dir_diffusion_blur(ctx, developed);
        SpkFilmCouplerApplyArgs aa{uint32_t(plane.pixels()), s.curves.K};
        {
            gpu::Batch bt = ctx.gpu.batch();
            bt.dispatch_1d(ctx.kernel("spk_film_coupler_apply"), aa.n,
                           {gpu::Arg::plane(plane), gpu::Arg::plane(developed), gpu::Arg::buffer(s.curve_buffer),
                            gpu::Arg::value(aa)});
            bt.commit_and_wait();
        }
    } else {
        plane = developed;
    }
    if (s.grain) fx::grain(ctx, plane, *s.grain, seed);
    gpu::Plane negative = ctx.gpu.persistent_plane(plane.w, plane.h, gpu::MemTag::Negative);
    std::memcpy(negative.data(), plane.data(), plane.bytes());
    return negative;
}

int32_t fail_status(const std::exception& e) {
    if (const auto* se = dynamic_cast<const Error*>(&e)) {
        last_error::set(se->what());
        return se->status();
    }
    last_error::set(e.what());
    return SPK_ERR_INTERNAL;
}

json::Value darr(const double* v, size_t n) {
    json::Array a;
    for (size_t i = 0; i < n; ++i) a.emplace_back(v[i]);
    return json::Value(std::move(a));
}

json::Value farr(const float* v, size_t n) {
    json::Array a;
    for (size_t i = 0; i < n; ++i) a.emplace_back(double(v[i]));
    return json::Value(std::move(a));
}

}  // namespace

extern "C" {

/* spkref_render(engine, rgb, w, h, delta, n, weights, sigmas, strength, exposures, n_prints, out_rgba, out_negative)
 *   open + develop (halation mixture in pixels when n > 0) + one print per entry of exposures
 *   (print_exposure values; the first is the render, the others reprints of the same negative)
 *   out_rgba: n_prints x h x w x 4 uint16, packed rows; out_negative: h x w x 3 floats or NULL
 *   film seed: the first draw of a fresh seed sequence when grain is on, else 0x5EED
 */
__attribute__((visibility("default"))) int32_t spkref_render(spk_engine* eng, const float* rgb, uint32_t w, uint32_t h,
                                                             const char* delta, uint32_t n, const double* weights,
                                                             const double* sigmas, const double* strength,
                                                             const double* exposures, uint32_t n_prints,
                                                             uint16_t* out_rgba, float* out_negative) {
    try {
        Engine& e = *reinterpret_cast<Engine*>(eng);
        Built b = build(e, delta);
        using params::P;
        gpu::Plane src = e.gpu().persistent_plane(w, h, gpu::MemTag::Source);
        float* o = src.data();
        for (size_t i = 0; i < size_t(w) * h * 3; ++i) o[i] = std::isfinite(rgb[i]) ? rgb[i] : 0.0f;
        core::RenderContext ctx{.gpu = e.gpu(), .device = e.device(), .variants = e.variants()};
        ctx.pitch_um = film::pitch_um(b.p->f(P::film_format_mm), std::max(w, h));
        ctx.rho_tier = 1.0;
        fx::SeedSequence seeds;
        const uint32_t seed = b.p->b(P::grain_active) ? seeds.next() : fx::kNoGrainFilmSeed;
        gpu::Plane neg = develop_override(ctx, *b.film, src, seed, n, weights, sigmas, strength);
        if (out_negative) std::memcpy(out_negative, neg.data(), neg.bytes());
        for (uint32_t k = 0; k < n_prints; ++k) {
            print::LiveParams live = print::LiveParams::from(*b.p);
            live.print_exposure = exposures[k];
            gpu::OutputImage img = print::print_scan_encode(ctx, *b.print, {neg, live, 0u});
            uint16_t* dst = out_rgba + size_t(k) * w * h * 4;
            for (uint32_t y = 0; y < h; ++y)
                std::memcpy(dst + size_t(y) * w * 4, img.rgba16 + size_t(y) * img.row_stride_px * 4, size_t(w) * 8);
            gpu::Context::release_texture(img.texture);
        }
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

/* A session-like handle for timing: spkref_open builds the set-up and copies the frame (what the
 * reference's spk_open does), spkref_develop and spkref_print are the render and the reprint. */
struct RefSession {
    Engine* e = nullptr;
    Built b;
    gpu::Plane src, neg;
    std::vector<double> weights, sigmas;
    double strength[3] = {0, 0, 0};
    uint32_t n = 0;
    fx::SeedSequence seeds;
};

__attribute__((visibility("default"))) void* spkref_open(spk_engine* eng, const float* rgb, uint32_t w, uint32_t h,
                                                         const char* delta, uint32_t n, const double* weights,
                                                         const double* sigmas, const double* strength) {
    try {
        auto* s = new RefSession();
        s->e = reinterpret_cast<Engine*>(eng);
        s->b = build(*s->e, delta);
        s->src = s->e->gpu().persistent_plane(w, h, gpu::MemTag::Source);
        float* o = s->src.data();
        for (size_t i = 0; i < size_t(w) * h * 3; ++i) o[i] = std::isfinite(rgb[i]) ? rgb[i] : 0.0f;
        s->n = n;
        s->weights.assign(weights, weights + 3 * n);
        s->sigmas.assign(sigmas, sigmas + 3 * n);
        for (int c = 0; c < 3; ++c) s->strength[c] = strength ? strength[c] : 0.0;
        return s;
    } catch (const std::exception& ex) {
        fail_status(ex);
        return nullptr;
    }
}

__attribute__((visibility("default"))) int32_t spkref_develop(void* handle) {
    try {
        auto* s = static_cast<RefSession*>(handle);
        using params::P;
        core::RenderContext ctx{.gpu = s->e->gpu(), .device = s->e->device(), .variants = s->e->variants()};
        ctx.pitch_um = film::pitch_um(s->b.p->f(P::film_format_mm), std::max(s->src.w, s->src.h));
        const uint32_t seed = s->b.p->b(P::grain_active) ? s->seeds.next() : fx::kNoGrainFilmSeed;
        s->neg = gpu::Plane{};
        s->neg = develop_override(ctx, *s->b.film, s->src, seed, s->n, s->weights.data(), s->sigmas.data(), s->strength);
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

__attribute__((visibility("default"))) int32_t spkref_print(void* handle, double print_exposure, uint16_t* out_rgba) {
    try {
        auto* s = static_cast<RefSession*>(handle);
        core::RenderContext ctx{.gpu = s->e->gpu(), .device = s->e->device(), .variants = s->e->variants()};
        ctx.pitch_um = film::pitch_um(s->b.p->f(params::P::film_format_mm), std::max(s->src.w, s->src.h));
        ctx.rho_tier = 1.0;
        print::LiveParams live = print::LiveParams::from(*s->b.p);
        live.print_exposure = print_exposure;
        gpu::OutputImage img = print::print_scan_encode(ctx, *s->b.print, {s->neg, live, 0u});
        if (out_rgba)
            for (uint32_t y = 0; y < s->neg.h; ++y)
                std::memcpy(out_rgba + size_t(y) * s->neg.w * 4, img.rgba16 + size_t(y) * img.row_stride_px * 4,
                            size_t(s->neg.w) * 8);
        gpu::Context::release_texture(img.texture);
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

__attribute__((visibility("default"))) void spkref_close(void* handle) { delete static_cast<RefSession*>(handle); }

/* spkref_meter(rgb, w, h, rgb_to_xyz, out7): the reference's meter statistics (src/film/meter.cpp:45-120)
 * of an image, in the order center_weighted, average, median, balanced, center, protect_highlights,
 * protect_shadows */
__attribute__((visibility("default"))) int32_t spkref_meter(const float* rgb, uint32_t w, uint32_t h,
                                                            const double* rgb_to_xyz, double* out) {
    try {
        res::Mat3 m{};
        for (size_t i = 0; i < 9; ++i) m[i] = rgb_to_xyz[i];
        const film::MeterValues v = film::meter_values(rgb, w, h, m);
        const double r[7] = {v.center_weighted, v.average, v.median, v.balanced, v.center, v.protect_highlights,
                             v.protect_shadows};
        std::memcpy(out, r, sizeof r);
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

/* spkref_downscale(rgb, w, h, long_edge, out, out_w, out_h): the reference's CPU tier downscale
 * (src/session/tiers.cpp:196-227) at a target long edge; out holds w h 3 floats */
__attribute__((visibility("default"))) int32_t spkref_downscale(const float* rgb, uint32_t w, uint32_t h,
                                                                uint32_t long_edge, float* out, uint32_t* out_w,
                                                                uint32_t* out_h) {
    try {
        const session::Size o = session::downscale_size(w, h, long_edge);
        session::downscale_cpu(rgb, w, h, out, o.w, o.h);
        *out_w = o.w;
        *out_h = o.h;
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

/* spkref_setup_json(engine, delta, pitch_um, out_json): the reference's narrowed kernel constants under the
 * same keys as the B200 build's spkx_session_setup_json */
__attribute__((visibility("default"))) int32_t spkref_setup_json(spk_engine* eng, const char* delta, double pitch_um,
                                                                 char** out_json) {
    try {
        Engine& e = *reinterpret_cast<Engine*>(eng);
        Built b = build(e, delta);
        const film::FilmSetup::Impl& f = b.film->impl();
        const print::PrintSetup::Impl& s = b.print->impl();
        json::Value r;
        r["input_matrix"] = farr(f.input_matrix_f32.data(), 9);
        r["L"] = f.table->size;
        r["table"] = farr(f.table->f32.as<float>(), f.table->f64.size());
        r["curve_x"] = farr(f.curves.x.data(), f.curves.x.size());
        r["curve_inv"] = farr(f.curves.inv.data(), f.curves.inv.size());
        r["curve_y"] = farr(f.curves.y.data(), f.curves.y.size());
        if (f.grain) {
            const fx::detail::GrainConstants kc = fx::detail::grain_constants(*f.grain, pitch_um);
            float cnt[9], sat[9], dml[9];
            for (int l = 0; l < 3; ++l)
                for (int c = 0; c < 3; ++c) {
                    cnt[3 * l + c] = num::f32(kc.count[l][c]);
                    sat[3 * l + c] = num::f32(kc.sat_d[l][c]);
                    dml[3 * l + c] = num::f32(kc.dmin_l[l][c]);
                }
            r["grain_count"] = farr(cnt, 9);
            r["grain_sat_d"] = farr(sat, 9);
            r["grain_dmin_l"] = farr(dml, 9);
        }
        const auto run = print::compute_run(s, print::LiveParams::from(*b.p));
        r["enl_eps"] = farr(run->enl.eps, 243);
        r["enl_beta"] = farr(run->enl.beta, 81);
        r["enl_wt"] = farr(run->enl.wt, 243);
        r["enl_g"] = farr(run->enl.g, 3);
        r["enl_o"] = farr(run->enl.o, 3);
        r["k_gain"] = double(run->k_gain);
        r["scan_eps"] = farr(s.scan_args.eps, 243);
        r["scan_beta"] = farr(s.scan_args.beta, 81);
        r["scan_wt"] = farr(s.scan_args.wt, 243);
        r["paper"] = farr(s.curve_gpu.as<float>(), size_t(s.curve_k) * 5);
        r["to_rgb"] = farr(s.to_rgb.m, 9);
        r["m_nid"] = farr(s.enc_args.m_nid, 9);
        const SpkPrintCam16Args& q = s.cam_args;
        const float cam[] = {q.f_l, q.n_bb, q.n_cb, q.n, q.z, q.a_w, q.c, q.n_c, q.j_first, q.j_last, q.h_first,
                             q.h_step, q.knee[0], q.knee[1], q.knee[2], q.lc[0], q.lc[1], q.lc[2], q.j_white,
                             q.d_rgb[0], q.d_rgb[1], q.d_rgb[2]};
        r["cam_k"] = farr(cam, 22);
        r["cam_m_to_xyz"] = farr(q.m_to_xyz, 9);
        r["cam_m_to_rgb"] = farr(q.m_to_rgb, 9);
        r["cmax"] = farr(s.cam->cmax_f32.data(), s.cam->cmax_f32.size());
        // the binary64 values behind the narrowed ones, where the reference keeps them
        json::Value f64;
        f64["table"] = darr(f.table->f64.data(), f.table->f64.size());
        f64["input_matrix"] = darr(f.input_matrix.data(), 9);
        f64["enl_eps"] = darr(run->eps_n.data(), run->eps_n.size());
        f64["enl_beta"] = darr(run->beta_n.data(), run->beta_n.size());
        f64["enl_wt"] = darr(run->w_n.data(), run->w_n.size());
        f64["enl_g"] = darr(run->g.data(), 3);
        f64["enl_o"] = darr(run->o.data(), 3);
        f64["scan_eps"] = darr(s.scan.eps.data(), s.scan.eps.size());
        f64["scan_beta"] = darr(s.scan.beta.data(), s.scan.beta.size());
        f64["scan_wt"] = darr(s.scan.wt.data(), s.scan.wt.size());
        f64["cmax"] = darr(s.cam->cmax_f64.data(), s.cam->cmax_f64.size());
        f64["cam_m_to_xyz"] = darr(s.cam->m_to_xyz.data(), 9);
        f64["cam_m_to_rgb"] = darr(s.cam->m_to_rgb.data(), 9);
        r["f64"] = std::move(f64);
        const std::string text = json::write(r);
        char* p = static_cast<char*>(std::malloc(text.size() + 1));
        std::memcpy(p, text.c_str(), text.size() + 1);
        *out_json = p;
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

/* spkref_sampler(engine, lam, counts, lognormal, n, stream, seed, mean, sd): the reference's
 * spk_fx_grain_test_sampler kernel (its Poisson and lognormal draws, host libm) */
__attribute__((visibility("default"))) int32_t spkref_sampler(spk_engine* eng, const float* lam, float* counts,
                                                              float* lognormal, uint32_t n, uint32_t stream,
                                                              uint32_t seed, float mean, float sd) {
    try {
        Engine& e = *reinterpret_cast<Engine*>(eng);
        gpu::Buffer bl = e.gpu().pool().acquire(size_t(n) * 4), bc = e.gpu().pool().acquire(size_t(n) * 4),
                    bg = e.gpu().pool().acquire(size_t(n) * 4);
        std::memcpy(bl.contents(), lam, size_t(n) * 4);
        struct {
            uint32_t n, stream, seed;
            float mean, stddev;
        } a{n, stream, seed, mean, sd};
        gpu::Batch bt = e.gpu().batch();
        bt.dispatch_1d(e.gpu().kernel("spk_fx_grain_test_sampler"), n,
                       {gpu::Arg::buffer(bl), gpu::Arg::buffer(bc), gpu::Arg::buffer(bg), gpu::Arg::value(a)});
        bt.commit_and_wait();
        std::memcpy(counts, bc.contents(), size_t(n) * 4);
        if (lognormal) std::memcpy(lognormal, bg.contents(), size_t(n) * 4);
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

/* spkref_gaussian(engine, in, out, w, h, sigma3, same_order_cpu): the reference's blur of a plane;
 * same_order_cpu = 1 runs its binary64-state host copy fx::cpu::gaussian instead of the kernels */
__attribute__((visibility("default"))) int32_t spkref_gaussian(spk_engine* eng, const float* in, float* out, uint32_t w,
                                                               uint32_t h, const double* sigma3, int32_t same_order_cpu) {
    try {
        const fx::Vec3 s{sigma3[0], sigma3[1], sigma3[2]};
        if (same_order_cpu) {
            fx::cpu::gaussian(in, out, w, h, s);
            return SPK_OK;
        }
        Engine& e = *reinterpret_cast<Engine*>(eng);
        core::RenderContext ctx{.gpu = e.gpu(), .device = e.device(), .variants = e.variants()};
        gpu::Plane a = ctx.scratch(w, h);
        std::memcpy(a.data(), in, a.bytes());
        gpu::Plane b;
        fx::gaussian(ctx, a, b, s);
        std::memcpy(out, b.data(), b.bytes());
        return SPK_OK;
    } catch (const std::exception& ex) {
        return fail_status(ex);
    }
}

}  // extern "C"
