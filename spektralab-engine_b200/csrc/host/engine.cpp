// Engine, session and every exported entry point of the B200 build.
//
// Behaviour mirrors the reference's session layer where the render path needs it
// (src/session/session.cpp: open :121-197, set_params :216-259, render/reprint :405-450, seeds
// :327-345; src/abi/abi.cpp: status mapping :40-65, result zeroing and scrubbing :84-92, :293-308).
// The device work is this build's own: one CUDA stream and one scratch pool per session, the source
// frame and the per-tier negatives resident in device memory, the result copied once to pinned host
// memory.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>

#include "../cuda/iir.hpp"
#include "../cuda/launch.hpp"
#include "device.hpp"
#include "render.hpp"
#include "spektralab.h"
#include "spektralab_b200.h"
#include "status.hpp"
#include "meter.hpp"
#include "tiers.hpp"

namespace spkb {

// ---- last error ----------------------------------------------------------------------------------
namespace last_error {
namespace {
thread_local std::string slot;
}
void set(const std::string& m) { slot = m; }
void clear() { slot.clear(); }
const char* get() { return slot.c_str(); }
}  // namespace last_error

namespace {

std::atomic<uint64_t> g_next_id{1};
constexpr uint64_t kMaxPixels = 151301008ull;

// splitmix64 seed sequence (reference src/fx/rng.hpp:17-41): one per pipeline, reset at every build.
struct SeedSequence {
    uint64_t state = 0x243F6A8885A308D3ull;
    uint32_t next() {
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z = z ^ (z >> 31);
        return uint32_t(z);
    }
};
constexpr uint32_t kNoGrainFilmSeed = 0x5EEDu;

enum class Tier { Live = 0, Preview = 1, Full = 2 };
std::optional<Tier> parse_tier(const char* s) {
    if (!s) return std::nullopt;
    const std::string t(s);
    if (t == "live") return Tier::Live;
    if (t == "preview") return Tier::Preview;
    if (t == "full") return Tier::Full;
    return std::nullopt;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

class Session;

class Engine {
public:
    int device = 0;
    std::shared_ptr<Resources> res;
    Cam16Cache cam16;
    std::mutex m;
    std::set<Session*> sessions;
    std::string capabilities, memory_report;
    // Built pipelines by parameter set: the binary64 set-up and its device tables depend only on the
    // parameters and the resources, so a later open or rebuild with the same parameters reuses them.
    std::mutex pipelines_m;
    std::vector<std::pair<std::string, Pipeline>> pipelines;  // most recent last
    // print-preview tables in device memory, by print stock (uploaded on first use, kept)
    std::mutex luts_m;
    std::map<std::string, DevBuffer> luts;
    static constexpr size_t kPipelineCache = 8;

    // Batched renders (spkx_render_batch): one at a time per engine, on their own streams. The plan chosen
    // for a list of frame sizes is kept, and so is the instantiated graph of each (plan, sizes) pair, which a
    // later batch of the same shape updates in place.
    std::mutex batch_m;
    cudaStream_t batch_stream = nullptr;
    std::vector<cudaStream_t> workers;
    std::vector<cudaEvent_t> frame_events;  // one per frame slot: completion, recorded inside the graph
    std::vector<cudaEvent_t> ready_events;  // one per frame slot: the frame's negative is ready
    std::vector<cudaEvent_t> join_events;   // one per worker stream
    cudaEvent_t fork_event = nullptr, start_event = nullptr;
    std::map<std::string, std::string> tuned;
    std::string pinned_plan;  // set by spkx_engine_batch_plan: used for every batch, no tuning
    std::map<std::string, cudaGraphExec_t> graphs;
    static constexpr size_t kGraphCache = 16;

    // A session's two streams and its row-band events, returned here when it is released and reused by
    // the next session (creating and destroying them cost an open-render-release cycle about 0.1 ms)
    struct SessionStreams {
        cudaStream_t stream = nullptr, copy = nullptr;
        std::vector<cudaEvent_t> band_events;
    };
    std::mutex streams_m;
    std::vector<SessionStreams> idle_streams;
    static constexpr size_t kIdleStreams = 16;

    SessionStreams take_streams() {
        {
            std::lock_guard<std::mutex> g(streams_m);
            if (!idle_streams.empty()) {
                SessionStreams t = std::move(idle_streams.back());
                idle_streams.pop_back();
                return t;
            }
        }
        SessionStreams t;
        cuda_check(cudaStreamCreateWithFlags(&t.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        const cudaError_t err = cudaStreamCreateWithFlags(&t.copy, cudaStreamNonBlocking);
        if (err != cudaSuccess) {
            cudaStreamDestroy(t.stream);
            cuda_check(err, "cudaStreamCreate");
        }
        return t;
    }
    // s's streams are idle (synchronised by the caller)
    void give_streams(SessionStreams s) {
        {
            std::lock_guard<std::mutex> g(streams_m);
            if (idle_streams.size() < kIdleStreams) {
                idle_streams.push_back(std::move(s));
                return;
            }
        }
        destroy_streams(s);
    }
    static void destroy_streams(SessionStreams& s) {
        for (cudaEvent_t e : s.band_events) cudaEventDestroy(e);
        if (s.copy) cudaStreamDestroy(s.copy);
        if (s.stream) cudaStreamDestroy(s.stream);
        s = SessionStreams{};
    }

    ~Engine() {
        for (SessionStreams& t : idle_streams) destroy_streams(t);
        if (batch_stream) cudaStreamSynchronize(batch_stream);
        for (auto& [k, g] : graphs) cudaGraphExecDestroy(g);
        for (cudaStream_t w : workers) cudaStreamDestroy(w);
        for (cudaEvent_t ev : frame_events) cudaEventDestroy(ev);
        for (cudaEvent_t ev : ready_events) cudaEventDestroy(ev);
        for (cudaEvent_t ev : join_events) cudaEventDestroy(ev);
        if (fork_event) cudaEventDestroy(fork_event);
        if (start_event) cudaEventDestroy(start_event);
        if (batch_stream) cudaStreamDestroy(batch_stream);
    }
};

struct TierState {
    Plane source;            // the tier's image (the frame itself when it fits the tier)
    uint32_t long_edge = 0;  // of the tier's image
    Plane negative;
    double pitch_um = 0.0;
    std::optional<double> applied_ev;  // the auto-exposure EV the negative was developed with
};

// The effect variants of the desktop device, the one this build serves (reference src/core/render.hpp:40-44)
constexpr const char* kEffectVersions =
    "halation=reference;grain=reference;glare=reference;print_spatial=reference;dir_couplers=reference";

// A session's progress record (reference src/session/progress.cpp): the current render's id, its node
// total and the nodes passed, the last node's label, done, the applied EV and the cancel flag. It has its
// own small lock, apart from the session's, so spk_progress and spk_cancel answer while a render runs.
class ProgressRecord final : public ProgressSink {
public:
    // a render-type call starts: new id, node total, stage "queued"; the cancel flag is cleared
    void reset(std::string id, uint32_t total) {
        std::lock_guard<std::mutex> g(m_);
        id_ = std::move(id);
        total_ = total;
        fired_ = 0;
        stage_ = "queued";
        done_ = false;
        ev_.reset();
        cancelled_.store(false);
    }
    void add_nodes(uint32_t n) {
        std::lock_guard<std::mutex> g(m_);
        total_ += n;
    }
    // between stages: a set cancel flag ends the render with SPK_ERR_CANCELLED; else the label is recorded
    void node(const char* label) override {
        if (cancelled_.load(std::memory_order_relaxed)) fail_cancelled();
        std::lock_guard<std::mutex> g(m_);
        stage_ = label;
        ++fired_;
    }
    void finish(bool done, std::optional<double> ev) {
        std::lock_guard<std::mutex> g(m_);
        done_ = done;
        ev_ = ev;
    }
    // spk_cancel: a NULL id, or the current one, cancels the current render
    void cancel(const char* id) {
        std::lock_guard<std::mutex> g(m_);
        if (!id || id_ == id) cancelled_.store(true);
    }
    // the spk_progress reply; an id that is given and is not the current one is SPK_ERR_USER
    json::Value snapshot(const char* id) const {
        std::lock_guard<std::mutex> g(m_);
        if (id && *id && id_ != id) fail_user("unknown progress id '" + std::string(id) + "'");
        json::Value r;
        r["auto_exposure_ev"] = ev_ ? json::Value(*ev_) : json::Value(nullptr);
        r["cancelled"] = cancelled_.load();
        r["done"] = done_;
        r["effect_versions"] = std::string(kEffectVersions);
        r["memory_pressure_critical"] = false;  // no memory-pressure source on this device
        r["node_times"] = json::Object{};
        r["pct"] = done_ ? 100.0 : total_ ? 100.0 * std::min(fired_, total_) / double(total_) : 0.0;
        r["progress_id"] = id_;
        r["stage"] = stage_;
        return r;
    }

private:
    mutable std::mutex m_;
    std::atomic<bool> cancelled_{false};
    std::string id_;
    std::string stage_ = "queued";
    uint32_t fired_ = 0, total_ = 0;
    bool done_ = false;
    std::optional<double> ev_;
};

class Session {
public:
    Engine* engine = nullptr;
    std::string id;
    std::mutex m;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;     // the result's copy to host memory, in row bands
    std::vector<cudaEvent_t> band_events;  // their events (grown by the print side as needed)
    Pool pool;
    bool product_defaults = false;
    Plane source;
    ParamSet params;
    std::shared_ptr<const Profile> film, print;
    Pipeline pipe;
    LiveParams live;
    SeedSequence seeds;
    TierState tiers[3];
    std::optional<HalationOverride> hal;
    int print_mode = -1;  // spkx_session_set_print_mode: -1 the binary32 print kernel, else a SpectralMode
    uint32_t print_bins = SPKB_NL;
    ProgressRecord progress;
    Plane meter_image;                // the frame at the meter's 1600 px long edge, kept
    std::optional<MeterValues> meter;  // until a field of the meter's key changes

    ~Session() {
        // stream-ordered buffers are freed on the stream, so they go before it does
        for (TierState& t : tiers) t = TierState{};
        meter_image = Plane{};
        source = Plane{};
        pipe = Pipeline{};
        // idle streams go back to the engine for the next session; a stream that reports an error is
        // destroyed with its events instead
        Engine::SessionStreams t{stream, copy_stream, std::move(band_events)};
        const bool idle = (!stream || cudaStreamSynchronize(stream) == cudaSuccess) &&
                          (!copy_stream || cudaStreamSynchronize(copy_stream) == cudaSuccess);
        if (idle && stream && copy_stream && engine) {
            engine->give_streams(std::move(t));
        } else {
            (void)cudaGetLastError();
            Engine::destroy_streams(t);
        }
    }

    void digest(ParamSet& p, const Profile& f) const {
        if (auto pack = engine->res->neutral_filters(p.s(P::print_stock), p.s(P::enlarger_illuminant), f)) {
            p.set(P::c_filter_neutral, (*pack)[0]);
            p.set(P::m_filter_neutral, (*pack)[1]);
            p.set(P::y_filter_neutral, (*pack)[2]);
        }
    }

    Pipeline build(const ParamSet& p, std::shared_ptr<const Profile> f, std::shared_ptr<const Profile> pr) {
        check_supported(p);
        const std::string key = json::write(p.to_json()) + (product_defaults ? "|pd" : "|");
        {
            std::lock_guard<std::mutex> g(engine->pipelines_m);
            for (auto& [k, pl] : engine->pipelines)
                if (k == key) return pl;
        }
        Pipeline pl;
        auto fs = build_film_setup(p, f, *engine->res);
        pl.print = build_print_setup(p, *fs, pr, *engine->res, engine->cam16, !product_defaults);
        pl.film = fs;
        upload_tables(pool, stream, pl);
        std::lock_guard<std::mutex> g(engine->pipelines_m);
        engine->pipelines.emplace_back(key, pl);
        if (engine->pipelines.size() > Engine::kPipelineCache) engine->pipelines.erase(engine->pipelines.begin());
        return pl;
    }

    // The tier's image, downscaled from the frame on first use and kept (reference
    // src/session/session.cpp:282-292, src/session/tiers.cpp:39-64): live at preview_long_edge, preview at
    // 3400 px, full the frame itself; a frame that fits the tier is its own tier image.
    TierState& tier_source(Tier t) {
        TierState& ts = tiers[int(t)];
        if (!ts.source) {
            uint32_t L = 0;
            if (t == Tier::Live) L = uint32_t(params.i(P::preview_long_edge));
            if (t == Tier::Preview) L = kPreviewLongEdge;
            ts.source = downscale(pool, stream, source, L);
            ts.long_edge = std::max(ts.source.w, ts.source.h);
        }
        return ts;
    }
    // The auto-exposure EV of the develops, or none when auto_exposure is off (reference
    // src/session/session.cpp:294-320): the meter runs once, on the live tier's image when that is the
    // 1600 px downscale already, else on its own downscale, and is kept until a meter-key field changes.
    std::optional<double> session_ev() {
        if (!params.b(P::auto_exposure)) return std::nullopt;
        return ensure_meter().ev(params.s(P::auto_exposure_method));
    }
    const MeterValues& ensure_meter() {
        if (!meter) {
            if (!meter_image) {
                const TierState& live = tiers[int(Tier::Live)];
                if (live.source && params.i(P::preview_long_edge) == int64_t(kMeterLongEdge))
                    meter_image = live.source;
                else
                    meter_image = downscale(pool, stream, source, kMeterLongEdge);
            }
            meter = spkb::meter(pool, stream, meter_image, params, pipe.film->input_space);
        }
        return *meter;
    }
    // The print seed of a render or reprint: the next draw of the seed sequence when the glare can draw,
    // even where its stage is skipped (scan_film), else 0 (reference src/session/session.cpp:339-344)
    uint32_t draw_print_seed() { return pipe.print->glare_draws() ? seeds.next() : 0u; }
    // rho_tier: the tier image's long edge over the frame's (never L / M: the floor can give L - 1)
    double rho(const TierState& ts) const { return double(ts.long_edge) / double(std::max(source.w, source.h)); }
    // the develop's pixel pitch at the tier's long edge
    double tier_pitch_um(const TierState& ts) const {
        return 1000.0 * params.f(P::film_format_mm) / double(ts.long_edge);
    }

    // a render-type call starts: a new progress id and the node total of its develop (unless the negative
    // is reused) and print
    std::string begin_progress(bool develops, bool prints = true) {
        uint32_t total = 0;
        if (develops && pipe.film) total += film_node_count(*pipe.film);
        if (prints && pipe.print) total += print_node_count(*pipe.print);
        std::string pid = "p" + std::to_string(g_next_id++);
        progress.reset(pid, total);
        return pid;
    }
};

namespace {

Engine* E(spk_engine* e) { return reinterpret_cast<Engine*>(e); }
Session* S(spk_session* s) { return reinterpret_cast<Session*>(s); }

int32_t map_exception() noexcept {
    try {
        throw;
    } catch (const Error& e) {
        last_error::set(e.what());
        return e.status();
    } catch (const std::bad_alloc&) {
        last_error::set("out of memory");
        return SPK_ERR_GPU;
    } catch (const std::exception& e) {
        last_error::set(std::string("internal error: ") + e.what());
        return SPK_ERR_INTERNAL;
    } catch (...) {
        last_error::set("internal error: unknown exception");
        return SPK_ERR_INTERNAL;
    }
}

template <class F>
int32_t guarded(F&& f) noexcept {
    try {
        return f();
    } catch (...) {
        return map_exception();
    }
}

int32_t invalid(const char* msg) noexcept {
    last_error::set(msg);
    return SPK_ERR_INVALID_ARG;
}

void put_json(char** out, const std::string& s) {
    if (!out) return;
    char* p = static_cast<char*>(std::malloc(s.size() + 1));
    if (!p) throw std::bad_alloc();
    std::memcpy(p, s.data(), s.size() + 1);
    *out = p;
}

void release_result(spk_result* r) {
    if (r->texture) output_release(static_cast<OutputImage*>(r->texture));
    std::memset(r, 0, sizeof *r);
}

std::string build_info_string() {
    return std::string("spektralab-native ") + SPK_VERSION_STRING + " (b200 sm_100a, math=safe)";
}

spk_engine* create(const char* dir, void* device, int32_t type) noexcept {
    last_error::clear();
    try {
        if (!dir) fail_invalid("resources_dir is NULL");
        if (type != SPK_DEVICE_DESKTOP)
            fail_user("device types PHONE and TABLET select mobile effect variants, which this B200 build does not have");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            (void)cudaGetLastError();
            fail_gpu("no CUDA device");
        }
        int dev = 0;
        if (device) dev = *static_cast<const int*>(device);
        else cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        if (dev < 0 || dev >= n) fail_gpu("CUDA device ordinal out of range");
        DeviceGuard g(dev);
        configure_device_pool(dev);
        dev::develop_prepare(nullptr);
        auto e = std::make_unique<Engine>();
        e->device = dev;
        e->res = Resources::load(dir);
        return reinterpret_cast<spk_engine*>(e.release());
    } catch (...) {
        map_exception();
        return nullptr;
    }
}

Session* open_session(Engine& e, const void* data, bool device_ptr, uint32_t w, uint32_t h, uint32_t ch,
                      const char* delta_text, std::string* reply) {
    if (ch != 3 && ch != 4) fail_user("input has " + std::to_string(ch) + " channels; expected 3 or 4");
    if (w == 0 || h == 0) fail_user("input has a zero width or height");
    const uint64_t npx = uint64_t(w) * h;
    if (npx > kMaxPixels)
        fail_user("input of " + std::to_string(w) + " x " + std::to_string(h) + " = " + std::to_string(npx) +
                  " pixels exceeds the cap of 151301008 pixels (14204 x 10652)");
    if (!data) fail_invalid(device_ptr ? "input->buffer is NULL" : "input->data is NULL");
    const Delta d = validate_delta(delta_text ? delta_text : "", DeltaContext::Open);
    DeviceGuard dg(e.device);
    auto s = std::make_unique<Session>();
    s->engine = &e;
    s->product_defaults = d.product_defaults.value_or(false);
    {
        Engine::SessionStreams t = e.take_streams();
        s->stream = t.stream;
        s->copy_stream = t.copy;
        s->band_events = std::move(t.band_events);
    }
    s->pool.set_stream(s->stream);
    ParamSet p;
    for (const auto& [fid, v] : d.fields)
        if (fid == size_t(P::film_stock) || fid == size_t(P::print_stock)) p.set(fid, v);
    auto film = e.res->profile(p.s(P::film_stock));
    auto print = e.res->profile(p.s(P::print_stock));
    s->digest(p, *film);
    p.set(P::output_color_space, "ProPhoto RGB");
    p.set(P::output_cctf_encoding, true);
    apply_delta(p, d);
    s->digest(p, *film);

    // the frame: raw upload, then channels and non-finite values fixed on the device
    s->source = Plane{s->pool.acquire(size_t(npx) * 12), w, h};
    const size_t raw_bytes = size_t(npx) * ch * sizeof(float);
    DevBuffer raw = s->pool.acquire(raw_bytes);
    cuda_check(cudaMemcpyAsync(raw.ptr(), data, raw_bytes, device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               s->stream),
               "frame upload");
    dev::source_copy(raw.as<float>(), s->source.data(), size_t(npx), ch, s->stream);
    cuda_check(cudaGetLastError(), "source copy");

    s->pipe = s->build(p, film, print);
    s->params = p;
    s->live = LiveParams::from(p);
    s->film = film;
    s->print = print;
    s->id = "s" + std::to_string(g_next_id++);
    cuda_check(cudaStreamSynchronize(s->stream), "open");
    if (reply) {
        json::Value r;
        json::Value meta;
        meta["width"] = w;
        meta["height"] = h;
        meta["megapixels"] = std::round(double(npx) / 1e4) / 100.0;
        meta["source"] = "<in-process>";
        r["meta"] = std::move(meta);
        json::Value di;
        di["input_cctf_decoding"] = s->params.b(P::input_cctf_decoding);
        di["input_color_space"] = s->params.s(P::input_color_space);
        di["input_color_space_source"] = "caller";
        r["detected_input"] = std::move(di);
        r["params"] = s->params.to_json();
        r["session_id"] = s->id;
        *reply = json::write(r);
    }
    Session* out = s.release();
    std::lock_guard<std::mutex> g(e.m);
    e.sessions.insert(out);
    return out;
}

// develop the tier (reference src/session/session.cpp:327-340): drop its negative, draw the film seed
void develop_tier(Session& s, Tier t, RenderCtx& ctx) {
    TierState& ts = s.tier_source(t);
    ts.negative = Plane{};
    ctx.ae_ev = s.session_ev();
    const uint32_t seed = s.params.b(P::grain_active) ? s.seeds.next() : kNoGrainFilmSeed;
    ctx.pitch_um = s.tier_pitch_um(ts);
    ts.applied_ev.reset();
    ts.negative = develop(ctx, s.pipe, ts.source, seed, s.hal);
    ts.pitch_um = ctx.pitch_um;
    ts.applied_ev = ctx.ae_ev;
}

void render(Session& s, const char* tier_name, bool reprint, spk_result* out) {
    std::lock_guard<std::mutex> lock(s.m);
    const auto t0 = std::chrono::steady_clock::now();
    const std::optional<Tier> t = parse_tier(tier_name);
    if (!t) fail_invalid(std::string("unknown tier '") + (tier_name ? tier_name : "") + "'");
    DeviceGuard dg(s.engine->device);
    TierState& ts = s.tiers[int(*t)];
    const bool reuse = reprint && static_cast<bool>(ts.negative);
    const std::string pid = s.begin_progress(!reuse);
    device_pool_begin_frame(s.engine->device);
    bool developed = false;
    OutputImage* img = nullptr;
    try {
        s.tier_source(*t);  // a failed downscale is a render failure (SPK_ERR_GPU), as in the reference
        RenderCtx ctx{s.pool, s.stream};
        ctx.progress = &s.progress;
        ctx.rho_tier = s.rho(ts);
        ctx.print_mode = s.print_mode;
        ctx.print_bins = s.print_bins;
        if (!reuse) {
            developed = true;
            develop_tier(s, *t, ctx);
        }
        ctx.print_seed = s.draw_print_seed();
        ctx.pitch_um = ts.pitch_um;
        img = output_acquire(s.engine->device, ts.negative.w, ts.negative.h);
        ctx.copy_stream = s.copy_stream;
        ctx.band_events = &s.band_events;
        if (!print_scan_encode(ctx, s.pipe, s.live, ts.negative, img, true))
            cuda_check(cudaMemcpyAsync(img->host, img->dev, img->bytes, cudaMemcpyDeviceToHost, s.stream),
                       "result copy");
        cuda_check(cudaStreamSynchronize(s.stream), "render");
        cuda_check(cudaGetLastError(), "render");
    } catch (...) {
        // band copies may still be writing the image's host pixels
        (void)cudaStreamSynchronize(s.copy_stream);
        (void)cudaStreamSynchronize(s.stream);
        if (img) output_release(img);
        if (developed) {  // a cancelled or failed render caches no negative of its own; a reused one stays
            ts.negative = Plane{};
            ts.applied_ev.reset();
        }
        s.progress.finish(false, std::nullopt);
        try {
            throw;
        } catch (const Error& e) {
            if (e.status() == SPK_ERR_CANCELLED || e.status() == SPK_ERR_INVALID_ARG) throw;
            fail_gpu(e.what());
        } catch (const std::bad_alloc&) {
            fail_gpu("out of memory");
        }
    }
    s.progress.finish(true, ts.applied_ev);
    out->rgba16 = img->host;
    out->texture = img;
    out->width = img->width;
    out->height = img->height;
    out->row_stride_px = img->stride_px;
    out->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    out->reprint = reuse ? 1 : 0;
    out->negative_was_cached = reuse ? 1 : 0;
    std::memset(out->progress_id, 0, sizeof out->progress_id);
    std::strncpy(out->progress_id, pid.c_str(), sizeof out->progress_id - 1);
}

// The print-preview table render (reference src/session/session.cpp:503-572): the tier's cached
// negative (developed and cached first when there is none, which draws the film seed but no print seed)
// through the stock's trilinear table into RGBA16. A missing table is SPK_ERR_USER before anything runs;
// the result always reads as a reprint of a cached negative.
void preview_stock_lut(Session& s, const char* print_stock, const char* tier_name, spk_result* out,
                       char** out_json) {
    std::lock_guard<std::mutex> lock(s.m);
    const auto t0 = std::chrono::steady_clock::now();
    const std::optional<Tier> t = parse_tier(tier_name ? tier_name : "live");
    if (!t) fail_invalid(std::string("unknown tier '") + tier_name + "'; expected live, preview or full");
    const std::string stock = print_stock && *print_stock ? std::string(print_stock) : s.params.s(P::print_stock);
    const std::shared_ptr<const PrintLut> lut = s.engine->res->print_lut(stock);
    DeviceGuard dg(s.engine->device);
    TierState& ts = s.tiers[int(*t)];
    const std::string pid = s.begin_progress(!ts.negative, false);  // the table pass is one more node
    s.progress.add_nodes(1);
    bool developed = false;
    OutputImage* img = nullptr;
    double apply_ms = 0.0;
    try {
        s.tier_source(*t);
        RenderCtx ctx{s.pool, s.stream};
        ctx.progress = &s.progress;
        ctx.rho_tier = s.rho(ts);
        if (!ts.negative) {
            developed = true;
            develop_tier(s, *t, ctx);
        }
        ctx.node("printing.preview_lut");
        DevBuffer table;
        {
            std::lock_guard<std::mutex> g(s.engine->luts_m);
            DevBuffer& d = s.engine->luts[stock];
            if (!d) {
                d = s.pool.persistent(lut->table.size() * sizeof(float));
                cuda_check(cudaMemcpy(d.ptr(), lut->table.data(), lut->table.size() * sizeof(float),
                                      cudaMemcpyHostToDevice),
                           "print table upload");
            }
            table = d;
        }
        img = output_acquire(s.engine->device, ts.negative.w, ts.negative.h);
        PrintLutArgs a{};
        a.lut = table.as<float>();
        a.size = lut->size;
        a.w = ts.negative.w;
        a.h = ts.negative.h;
        a.stride = img->stride_px;
        for (int c = 0; c < 3; ++c) {
            a.lo[c] = lut->lo[c];
            a.s[c] = f32(1.0 / (double(lut->hi[c]) - double(lut->lo[c])));
        }
        const auto ta = std::chrono::steady_clock::now();
        dev::print_lut(ts.negative.data(), img->dev, a, s.stream);
        cuda_check(cudaMemcpyAsync(img->host, img->dev, img->bytes, cudaMemcpyDeviceToHost, s.stream), "result copy");
        cuda_check(cudaStreamSynchronize(s.stream), "print table");
        cuda_check(cudaGetLastError(), "print table");
        apply_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta).count();
    } catch (...) {
        (void)cudaStreamSynchronize(s.stream);
        if (img) output_release(img);
        if (developed) {  // a cancelled or failed render caches no negative of its own; a reused one stays
            ts.negative = Plane{};
            ts.applied_ev.reset();
        }
        s.progress.finish(false, std::nullopt);
        try {
            throw;
        } catch (const Error& e) {
            if (e.status() == SPK_ERR_CANCELLED || e.status() == SPK_ERR_INVALID_ARG) throw;
            fail_gpu(e.what());
        } catch (const std::bad_alloc&) {
            fail_gpu("out of memory");
        }
    }
    s.progress.finish(true, ts.applied_ev);
    out->rgba16 = img->host;
    out->texture = img;
    out->width = img->width;
    out->height = img->height;
    out->row_stride_px = img->stride_px;
    out->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    out->reprint = 1;
    out->negative_was_cached = 1;
    std::memset(out->progress_id, 0, sizeof out->progress_id);
    std::strncpy(out->progress_id, pid.c_str(), sizeof out->progress_id - 1);
    if (out_json) {
        json::Value r;
        r["apply_backend"] = "native-cuda";
        r["apply_ms"] = apply_ms;
        r["declared_pairing"] = lut->declared_pairing;
        r["lut_source"] = "shipped";
        r["paired_film"] = lut->paired_film;
        r["print_stock"] = stock;
        r["tier"] = *t == Tier::Live ? "live" : (*t == Tier::Preview ? "preview" : "full");
        const std::string& film = s.params.s(P::film_stock);
        if (film != lut->paired_film)
            r["warning"] = "the print table for '" + stock + "' was made for '" + lut->paired_film + "', not for '" +
                           film + "'";
        put_json(out_json, json::write(r));
    }
}

spk_status render_common(spk_session* session, const char* tier, spk_result* out, bool reprint) {
    last_error::clear();
    if (!session) return invalid("session is NULL");
    if (!out) return invalid("out is NULL");
    if (!parse_tier(tier)) {
        last_error::set(std::string("unknown tier '") + (tier ? tier : "") + "'; expected live, preview or full");
        return SPK_ERR_INVALID_ARG;
    }
    std::memset(out, 0, sizeof *out);
    const int32_t st = guarded([&] {
        render(*S(session), tier, reprint, out);
        return SPK_OK;
    });
    if (st != SPK_OK) release_result(out);
    return st;
}

// ---- batched renders ------------------------------------------------------------------------------
//
// A batch renders many sessions' frames with one call. The film side of each frame runs on its session's
// stream as in spk_render (sessions develop concurrently); the print side and the scanner of every frame
// whose scanner takes the tiled kernel go into ONE CUDA graph on the engine's batch stream. Two plan
// families build that graph:
//   frames:K          each frame's print and scanner launches on one of K worker streams (round robin),
//                     forked from and joined to the batch stream; the frames overlap on the device;
//   persistent:S:C    one print launch and one scanner launch for all frames: C CTAs walking items of S
//                     pixels (print) and the frames' concatenated 32 x 32 tile lists (scanner);
//   persistent:S:C:G  the same launches for G consecutive groups of frames (about equal pixels each), each
//                     group's result copies on a worker stream while the next group's launches run.
// Every plan runs the same per-pixel and per-tile code as spk_render, so the pixels are those of singles.
// The first batch of a list of frame sizes times each candidate plan on the device and keeps the fastest.

struct BatchFrame {
    Session* s = nullptr;
    OutputImage* img = nullptr;
    Plane rgb;
    const float* neg = nullptr;
    PrintArgs pa{};
    Plane glare;             // the print glare's field (empty without glare)
    ScanArgs sa{};
    bool fused = false;      // print and scanner inside the batch graph
    bool reused = false;     // the tier's negative was cached (reprint)
    bool developed = false;  // the tier's negative was made by this batch
    cudaEvent_t ready = nullptr;  // the engine's ready event of the frame's slot
    std::string pid;              // the frame's progress id
};

// The tuner's candidates: per-frame launches on 4 or 16 streams, the persistent launches over a grid of item
// sizes (pixels per print item) and CTA counts (4, 8 and 16 per SM), and grouped persistent launches
const char* const kBatchPlans[] = {"frames:4",
                                   "frames:16",
                                   "persistent:2048:592",
                                   "persistent:2048:1184",
                                   "persistent:2048:2368",
                                   "persistent:8192:592",
                                   "persistent:8192:1184",
                                   "persistent:8192:2368",
                                   "persistent:32768:592",
                                   "persistent:32768:1184",
                                   "persistent:32768:2368",
                                   "persistent:8192:1184:4",
                                   "persistent:8192:1184:8",
                                   "persistent:8192:1184:16",
                                   "persistent:8192:2368:8",
                                   "persistent:32768:1184:8",
                                   "persistent:2048:1184:8"};
constexpr size_t kMaxWorkers = 16;

// A plan string: "frames:K" (1 <= K <= 16) or "persistent:S:C[:G]" (S even, 2 .. 2^20 pixels; 1 <= C <= 65535;
// 1 <= G <= 1024).
bool valid_plan(const std::string& p) {
    auto number = [](const std::string& t, unsigned long lo, unsigned long hi, unsigned long& v) {
        if (t.empty() || t.size() > 9 || t.find_first_not_of("0123456789") != std::string::npos) return false;
        v = std::stoul(t);
        return v >= lo && v <= hi;
    };
    unsigned long a = 0, b = 0;
    if (p.rfind("frames:", 0) == 0) return number(p.substr(7), 1, kMaxWorkers, a);
    if (p.rfind("persistent:", 0) != 0) return false;
    const std::string rest = p.substr(11);
    const size_t c = rest.find(':');
    if (c == std::string::npos) return false;
    const size_t c2 = rest.find(':', c + 1);
    unsigned long g = 1;
    if (c2 != std::string::npos && !number(rest.substr(c2 + 1), 1, 1024, g)) return false;
    return number(rest.substr(0, c), 2, 1ul << 20, a) && a % 2 == 0 &&
           number(rest.substr(c + 1, c2 == std::string::npos ? std::string::npos : c2 - c - 1), 1, 65535, b);
}

void batch_resources(Engine& e, size_t n_frames, size_t n_workers) {
    if (!e.batch_stream) cuda_check(cudaStreamCreateWithFlags(&e.batch_stream, cudaStreamNonBlocking), "batch stream");
    if (!e.fork_event) cuda_check(cudaEventCreateWithFlags(&e.fork_event, cudaEventDisableTiming), "batch event");
    if (!e.start_event) cuda_check(cudaEventCreate(&e.start_event), "batch event");
    while (e.workers.size() < n_workers) {
        cudaStream_t w = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking), "batch worker stream");
        e.workers.push_back(w);
        cudaEvent_t j = nullptr;
        cuda_check(cudaEventCreateWithFlags(&j, cudaEventDisableTiming), "batch event");
        e.join_events.push_back(j);
    }
    while (e.frame_events.size() < n_frames) {
        cudaEvent_t ev = nullptr;
        cuda_check(cudaEventCreate(&ev), "batch event");
        e.frame_events.push_back(ev);
    }
    while (e.ready_events.size() < n_frames) {
        cudaEvent_t ev = nullptr;
        cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "batch event");
        e.ready_events.push_back(ev);
    }
}

// Captures body(batch_stream) into a graph, brings the engine's executable graph for `key` up to date
// (updated in place when the topology is unchanged, else instantiated afresh) and launches it, between
// the timing events t0 and t1 when given.
template <class F>
void launch_captured(Engine& e, const std::string& key, F&& body, cudaEvent_t t0 = nullptr, cudaEvent_t t1 = nullptr) {
    cudaStream_t bs = e.batch_stream;
    cuda_check(cudaStreamBeginCapture(bs, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
        body(bs);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(bs, &g);
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        throw;
    }
    cudaGraph_t graph = nullptr;
    cuda_check(cudaStreamEndCapture(bs, &graph), "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    auto it = e.graphs.find(key);
    if (it != e.graphs.end()) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(it->second, graph, &info) == cudaSuccess) {
            exec = it->second;
        } else {
            (void)cudaGetLastError();
            cudaGraphExecDestroy(it->second);
            e.graphs.erase(it);
        }
    }
    if (!exec) {
        const cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
        if (err != cudaSuccess) {
            cudaGraphDestroy(graph);
            cuda_check(err, "cudaGraphInstantiate");
        }
        if (e.graphs.size() >= Engine::kGraphCache) {
            cudaGraphExecDestroy(e.graphs.begin()->second);
            e.graphs.erase(e.graphs.begin());
        }
        e.graphs[key] = exec;
    }
    cudaGraphDestroy(graph);
    if (t0) cuda_check(cudaEventRecord(t0, bs), "graph timing");
    cuda_check(cudaGraphLaunch(exec, bs), "cudaGraphLaunch");
    if (t1) cuda_check(cudaEventRecord(t1, bs), "graph timing");
}

// Enqueues the print side of the fused frames under `plan` on the batch stream (graph launch and, for the
// persistent plans, the upload of the frame tables before it). Each fused frame's result is copied to its
// pinned host image inside the graph, and frame_events[slot] marks its completion. In the per-frame plans
// each frame waits inside the graph for its own negative (its ready event), so a frame prints while
// later frames still develop; the persistent plans wait for every negative before their launch. The
// graph launch is bracketed by t0 and t1 when given.
void run_plan(Engine& e, const std::string& plan, const std::string& shape, std::vector<BatchFrame>& fr,
              const std::vector<size_t>& slots, DevBuffer& tables, cudaEvent_t t0 = nullptr, cudaEvent_t t1 = nullptr) {
    cudaStream_t bs = e.batch_stream;
    const std::string key = plan + "|" + shape;
    if (plan.rfind("frames:", 0) == 0) {
        const size_t K = std::min<size_t>(std::stoul(plan.substr(7)), std::max<size_t>(slots.size(), 1));
        launch_captured(
            e, key,
            [&](cudaStream_t s) {
                cuda_check(cudaEventRecord(e.fork_event, s), "fork");
                for (size_t k = 0; k < K; ++k) cuda_check(cudaStreamWaitEvent(e.workers[k], e.fork_event, 0), "fork");
                for (size_t j = 0; j < slots.size(); ++j) {
                    BatchFrame& f = fr[slots[j]];
                    cudaStream_t ws = e.workers[j % K];
                    cuda_check(cudaStreamWaitEvent(ws, f.ready, cudaEventWaitExternal), "frame ready");
                    dev::print(f.neg, f.rgb.data(), f.pa, ws);
                    dev::scan_encode(f.rgb.data(), f.img->dev, f.rgb.w, f.rgb.h, f.sa, ws);
                    cuda_check(cudaMemcpyAsync(f.img->host, f.img->dev, f.img->bytes, cudaMemcpyDeviceToHost, ws),
                               "result copy");
                    cuda_check(cudaEventRecordWithFlags(e.frame_events[slots[j]], ws, cudaEventRecordExternal), "frame");
                }
                for (size_t k = 0; k < K; ++k) {
                    cuda_check(cudaEventRecord(e.join_events[k], e.workers[k]), "join");
                    cuda_check(cudaStreamWaitEvent(s, e.join_events[k], 0), "join");
                }
            },
            t0, t1);
        return;
    }
    for (size_t slot : slots) cuda_check(cudaStreamWaitEvent(bs, fr[slot].ready, 0), "frame ready");
    // persistent:S:C[:G]
    const size_t c1 = plan.find(':'), c2 = plan.find(':', c1 + 1), c3 = plan.find(':', c2 + 1);
    const uint32_t item_px = uint32_t(std::stoul(plan.substr(c1 + 1, c2 - c1 - 1)));
    const uint32_t ctas = uint32_t(std::stoul(plan.substr(c2 + 1, c3 == std::string::npos ? std::string::npos : c3 - c2 - 1)));
    const size_t n = slots.size();
    const size_t G = std::min(n, c3 == std::string::npos ? size_t(1) : size_t(std::stoul(plan.substr(c3 + 1))));
    // the frames in G consecutive groups of about equal pixel counts
    std::vector<size_t> first(1, 0);
    {
        uint64_t total = 0, acc = 0;
        for (size_t slot : slots) total += fr[slot].pa.n;
        for (size_t j = 0; j < n && first.size() < G; ++j) {
            acc += fr[slots[j]].pa.n;
            if (acc * G >= total * first.size() && j + 1 < n) first.push_back(j + 1);
        }
        first.push_back(n);
    }
    // one table blob for all groups: per group its print frames, scanner frames and print items
    struct GroupLayout {
        size_t o_pf, o_sf, o_if, o_ip;
        uint32_t n_items, tiles;
        int r1, r2;
        bool shared;
    };
    auto up16 = [](size_t b) { return (b + 15) / 16 * 16; };
    std::vector<GroupLayout> gl(first.size() - 1);
    std::vector<unsigned char> blob;
    auto append = [&](const void* src, size_t bytes) {
        const size_t o = blob.size();
        blob.resize(o + up16(bytes), 0);
        if (bytes) std::memcpy(blob.data() + o, src, bytes);
        return o;
    };
    for (size_t g = 0; g + 1 < first.size(); ++g) {
        const size_t j0 = first[g], j1 = first[g + 1];
        std::vector<BatchPrintFrame> pf(j1 - j0);
        std::vector<BatchScanFrame> sf(j1 - j0);
        std::vector<uint32_t> item_frame, item_first;
        GroupLayout& L = gl[g];
        L.tiles = 0;
        L.r1 = fr[slots[j0]].sa.r1;
        L.r2 = fr[slots[j0]].sa.r2;
        // frames of the same stocks and filters share their spectral tables: the kernel then takes them once
        L.shared = true;
        for (size_t j = j0; j < j1; ++j) {
            BatchFrame& f = fr[slots[j]];
            pf[j - j0].args = f.pa;
            pf[j - j0].neg = f.neg;
            pf[j - j0].rgb = f.rgb.data();
            for (uint32_t q = 0; q < f.pa.n; q += item_px) {
                item_frame.push_back(uint32_t(j - j0));
                item_first.push_back(q);
            }
            sf[j - j0].args = f.sa;
            sf[j - j0].rgb = f.rgb.data();
            sf[j - j0].out = f.img->dev;
            sf[j - j0].w = f.rgb.w;
            sf[j - j0].h = f.rgb.h;
            sf[j - j0].tiles_x = dev::scan_tiles_x(f.rgb.w);
            sf[j - j0].first_tile = L.tiles;
            L.tiles += dev::scan_tiles(f.rgb.w, f.rgb.h);
            if (f.sa.r1 != L.r1 || f.sa.r2 != L.r2) L.r1 = L.r2 = -1;
            const PrintArgs& a0 = fr[slots[j0]].pa;
            L.shared = L.shared && std::memcmp(&f.pa.enl, &a0.enl, sizeof a0.enl) == 0 &&
                       std::memcmp(&f.pa.scan, &a0.scan, sizeof a0.scan) == 0;
        }
        L.n_items = uint32_t(item_frame.size());
        L.o_pf = append(pf.data(), pf.size() * sizeof(BatchPrintFrame));
        L.o_sf = append(sf.data(), sf.size() * sizeof(BatchScanFrame));
        L.o_if = append(item_frame.data(), item_frame.size() * sizeof(uint32_t));
        L.o_ip = append(item_first.data(), item_first.size() * sizeof(uint32_t));
    }
    Pool pool(bs);
    tables = pool.acquire(blob.size());
    unsigned char* d = tables.as<unsigned char>();
    cuda_check(cudaMemcpyAsync(d, blob.data(), blob.size(), cudaMemcpyHostToDevice, bs), "batch tables");
    // the pageable source is staged before cudaMemcpyAsync returns, so blob may go at scope exit
    const size_t K = std::min(gl.size(), kMaxWorkers);
    launch_captured(
        e, key,
        [&](cudaStream_t s) {
            for (size_t g = 0; g < gl.size(); ++g) {
                const GroupLayout& L = gl[g];
                const BatchFrame& f0 = fr[slots[first[g]]];
                dev::print_batch(reinterpret_cast<const BatchPrintFrame*>(d + L.o_pf),
                                 reinterpret_cast<const uint32_t*>(d + L.o_if),
                                 reinterpret_cast<const uint32_t*>(d + L.o_ip), L.n_items, item_px, ctas,
                                 L.shared ? &f0.pa.enl : nullptr, L.shared ? &f0.pa.scan : nullptr, s);
                dev::scan_encode_batch(reinterpret_cast<const BatchScanFrame*>(d + L.o_sf),
                                       uint32_t(first[g + 1] - first[g]), L.tiles, L.r1, L.r2, ctas, s);
                // one group: its copies follow on the batch stream; several: the group's copies run on a
                // worker stream while the next group's launches run
                cudaStream_t cs = s;
                if (gl.size() > 1) {
                    cs = e.workers[g % K];
                    cuda_check(cudaEventRecord(e.fork_event, s), "fork");
                    cuda_check(cudaStreamWaitEvent(cs, e.fork_event, 0), "fork");
                }
                for (size_t j = first[g]; j < first[g + 1]; ++j) {
                    BatchFrame& f = fr[slots[j]];
                    cuda_check(cudaMemcpyAsync(f.img->host, f.img->dev, f.img->bytes, cudaMemcpyDeviceToHost, cs),
                               "result copy");
                    cuda_check(cudaEventRecordWithFlags(e.frame_events[slots[j]], cs, cudaEventRecordExternal),
                               "frame");
                }
            }
            if (gl.size() > 1)
                for (size_t k = 0; k < K; ++k) {
                    cuda_check(cudaEventRecord(e.join_events[k], e.workers[k]), "join");
                    cuda_check(cudaStreamWaitEvent(s, e.join_events[k], 0), "join");
                }
        },
        t0, t1);
}

void render_batch(std::vector<Session*> ss, const char* tier_name, bool reprint, spk_result* out, std::string* info) {
    const std::optional<Tier> t = parse_tier(tier_name);
    if (!t) fail_invalid(std::string("unknown tier '") + (tier_name ? tier_name : "") + "'; expected live, preview or full");
    if (ss.empty()) fail_invalid("a batch needs at least one session");
    Engine& e = *ss[0]->engine;
    {
        std::vector<Session*> order = ss;
        std::sort(order.begin(), order.end());
        for (size_t i = 0; i < order.size(); ++i) {
            if (!order[i]) fail_invalid("a session of the batch is NULL");
            if (i && order[i] == order[i - 1]) fail_invalid("a session appears twice in the batch");
            if (order[i]->engine != &e) fail_invalid("the sessions of a batch must share one engine");
        }
    }
    // sessions locked in address order (no lock-order cycle with other batches), then the engine's batch
    std::vector<Session*> order = ss;
    std::sort(order.begin(), order.end());
    std::vector<std::unique_lock<std::mutex>> locks;
    locks.reserve(order.size());
    for (Session* s : order) locks.emplace_back(s->m);
    std::lock_guard<std::mutex> bl(e.batch_m);
    DeviceGuard dg(e.device);

    const size_t n = ss.size();
    std::vector<BatchFrame> fr(n);
    DevBuffer tables;
    std::string plan;
    double tuning_ms = 0.0;
    json::Value candidates = json::Object{};  // the timed plans of a tuning pass: device ms each
    std::vector<double> done_ms(n, 0.0);
    try {
        batch_resources(e, n, kMaxWorkers);
        dev::scan_prepare();
        cudaStream_t bs = e.batch_stream;
        const auto t0 = std::chrono::steady_clock::now();
        cuda_check(cudaEventRecord(e.start_event, bs), "batch start");
        std::vector<size_t> slots;
        std::string shape = std::string(tier_name);
        for (size_t i = 0; i < n; ++i) {
            Session& s = *ss[i];
            BatchFrame& f = fr[i];
            f.s = &s;
            TierState& ts = s.tiers[int(*t)];
            f.reused = reprint && static_cast<bool>(ts.negative);
            f.pid = s.begin_progress(!f.reused);
            s.tier_source(*t);
            RenderCtx ctx{s.pool, s.stream};
            ctx.progress = &s.progress;
            ctx.rho_tier = s.rho(ts);
            ctx.print_mode = s.print_mode;
            ctx.print_bins = s.print_bins;
            if (!f.reused) {
                f.developed = true;
                develop_tier(s, *t, ctx);
            }
            ctx.print_seed = s.draw_print_seed();
            ctx.pitch_um = ts.pitch_um;
            const uint32_t nw = ts.negative.w, nh = ts.negative.h;
            f.img = output_acquire(e.device, nw, nh);
            f.neg = ts.negative.data();
            // a session on the spectral-mode print kernel stays on its own stream
            f.fused = s.print_mode < 0 && scan_args(s.pipe, ctx.rho_tier, nw, nh, f.img->stride_px, f.sa);
            if (f.fused) {
                print_nodes(ctx, *s.pipe.print);
                f.pa = print_args(s.pipe, s.live, uint32_t(ts.negative.pixels()));
                f.glare = glare_plane(ctx, s.pipe, nw, nh);  // on the session's stream, before its ready event
                f.pa.glare = f.glare ? f.glare.data() : nullptr;
                f.rgb = make_plane(s.pool, nw, nh);
                f.ready = e.ready_events[i];
                cuda_check(cudaEventRecord(f.ready, s.stream), "frame ready");
                slots.push_back(i);
                shape += "," + std::to_string(nw) + "x" + std::to_string(nh);
            } else {
                // the scanner's separate passes: the frame stays on its session's stream
                print_scan_encode(ctx, s.pipe, s.live, ts.negative, f.img);
                cuda_check(cudaMemcpyAsync(f.img->host, f.img->dev, f.img->bytes, cudaMemcpyDeviceToHost, s.stream),
                           "result copy");
                cuda_check(cudaEventRecord(e.frame_events[i], s.stream), "frame");
            }
        }
        if (!slots.empty()) {
            auto tuned = e.tuned.find(shape);
            if (!e.pinned_plan.empty()) {
                plan = e.pinned_plan;
            } else if (tuned != e.tuned.end()) {
                plan = tuned->second;
            } else {
                // every candidate renders the whole batch; the pixels agree, so the last run's stand. The
                // negatives are complete first, so that each candidate's time is its graph's alone.
                for (size_t slot : slots) cuda_check(cudaEventSynchronize(fr[slot].ready), "frame ready");
                cudaEvent_t a = nullptr, b = nullptr;
                cuda_check(cudaEventCreate(&a), "batch event");
                cuda_check(cudaEventCreate(&b), "batch event");
                float best = 0.0f;
                try {
                    for (const char* cand : kBatchPlans) {
                        DevBuffer tb;
                        run_plan(e, cand, shape, fr, slots, tb, a, b);
                        cuda_check(cudaEventSynchronize(b), "tuning");
                        float ms = 0.0f;
                        cuda_check(cudaEventElapsedTime(&ms, a, b), "tuning");
                        tuning_ms += ms;
                        candidates[cand] = double(ms);
                        if (plan.empty() || ms < best) {
                            best = ms;
                            plan = cand;
                        }
                    }
                } catch (...) {
                    cudaEventDestroy(a);
                    cudaEventDestroy(b);
                    throw;
                }
                cudaEventDestroy(a);
                cudaEventDestroy(b);
                e.tuned[shape] = plan;
            }
            run_plan(e, plan, shape, fr, slots, tables);
        }
        cuda_check(cudaStreamSynchronize(bs), "batch");
        for (size_t i = 0; i < n; ++i) {
            cuda_check(cudaStreamSynchronize(ss[i]->stream), "batch");
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, e.start_event, e.frame_events[i]) == cudaSuccess) {
                done_ms[i] = ms;
            } else {
                (void)cudaGetLastError();
                done_ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            }
        }
        cuda_check(cudaGetLastError(), "batch");
    } catch (...) {
        if (e.batch_stream) (void)cudaStreamSynchronize(e.batch_stream);
        for (BatchFrame& f : fr) {
            if (f.s) (void)cudaStreamSynchronize(f.s->stream);
            if (f.img) output_release(f.img);
            f.img = nullptr;
            if (f.s) f.s->progress.finish(false, std::nullopt);
            if (f.developed) {
                f.s->tiers[int(*t)].negative = Plane{};
                f.s->tiers[int(*t)].applied_ev.reset();
            }
        }
        try {
            throw;
        } catch (const Error& err) {
            if (err.status() == SPK_ERR_CANCELLED || err.status() == SPK_ERR_INVALID_ARG) throw;
            fail_gpu(err.what());
        } catch (const std::bad_alloc&) {
            fail_gpu("out of memory");
        }
    }
    json::Value r;
    json::Array dms;
    for (size_t i = 0; i < n; ++i) {
        BatchFrame& f = fr[i];
        Session& s = *f.s;
        s.progress.finish(true, s.tiers[int(*t)].applied_ev);
        spk_result& o = out[i];
        o.rgba16 = f.img->host;
        o.texture = f.img;
        o.width = f.img->width;
        o.height = f.img->height;
        o.row_stride_px = f.img->stride_px;
        o.elapsed_ms = done_ms[i];
        o.reprint = f.reused ? 1 : 0;
        o.negative_was_cached = f.reused ? 1 : 0;
        std::memset(o.progress_id, 0, sizeof o.progress_id);
        std::strncpy(o.progress_id, f.pid.c_str(), sizeof o.progress_id - 1);
        dms.push_back(json::Value(done_ms[i]));
    }
    r["plan"] = plan.empty() ? std::string("none") : plan;
    r["tuning_ms"] = tuning_ms;
    if (!candidates.as_object().empty()) r["candidates_ms"] = std::move(candidates);
    r["frame_done_ms"] = json::Value(std::move(dms));
    if (info) *info = json::write(r);
}

}  // namespace

// ---- internal entry points used by the extension functions ---------------------------------------

std::string session_profile(Session& s, const char* tier_name, bool reprint, uint32_t steps) {
    std::lock_guard<std::mutex> lock(s.m);
    const std::optional<Tier> t = parse_tier(tier_name);
    if (!t) fail_invalid("unknown tier");
    DeviceGuard dg(s.engine->device);
    TierState& ts = s.tier_source(*t);
    DevBuffer flush = s.pool.acquire(size_t(256) << 20);
    OutputImage* img = nullptr;  // acquired at the negative's size (a geometry changes it)
    json::Value stages = json::Object{};
    json::Value kernels = json::Object{};
    json::Array totals;
    Timer timer;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const uint64_t launches0 = dev::launch_count();
    uint64_t flushes = 0;
    struct HookGuard {
        ~HookGuard() { dev::set_launch_hook(nullptr); }
    } hook_guard;
    try {
        for (uint32_t k = 0; k < steps; ++k) {
            dev::set_launch_hook(nullptr);
            dev::fill(flush.ptr(), flush.size() / 16 * 16, k, s.stream);
            ++flushes;
            dev::set_launch_hook(&timer);
            RenderCtx ctx{s.pool, s.stream};
            ctx.timer = &timer;
            ctx.rho_tier = s.rho(ts);
            ctx.print_mode = s.print_mode;
            ctx.print_bins = s.print_bins;
            cudaEventRecord(a, s.stream);
            if (!reprint || !ts.negative) {
                ctx.ae_ev = s.session_ev();
                ctx.pitch_um = s.tier_pitch_um(ts);
                const uint32_t seed = s.params.b(P::grain_active) ? s.seeds.next() : kNoGrainFilmSeed;
                ts.negative = develop(ctx, s.pipe, ts.source, seed, s.hal);
                ts.pitch_um = ctx.pitch_um;
            }
            ctx.print_seed = s.draw_print_seed();
            ctx.pitch_um = ts.pitch_um;
            if (!img) img = output_acquire(s.engine->device, ts.negative.w, ts.negative.h);
            print_scan_encode(ctx, s.pipe, s.live, ts.negative, img);
            cudaEventRecord(b, s.stream);
            cuda_check(cudaStreamSynchronize(s.stream), "profile step");
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            totals.push_back(json::Value(double(ms)));
            for (const Timer::Mark& m : timer.marks) {
                float sm = 0;
                cudaEventElapsedTime(&sm, m.a, m.b);
                json::Value& arr = stages[m.name];
                if (arr.is_null()) arr = json::Array{};
                arr.as_array().push_back(json::Value(double(sm)));
            }
            for (const Timer::Mark& m : timer.kernels) {
                float sm = 0;
                cudaEventElapsedTime(&sm, m.a, m.b);
                json::Value& arr = kernels[m.name];
                if (arr.is_null()) arr = json::Array{};
                arr.as_array().push_back(json::Value(double(sm)));
            }
            timer.reset();
        }
    } catch (...) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (img) output_release(img);
        throw;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (img) output_release(img);
    json::Value r;
    r["steps"] = steps;
    r["total_ms"] = std::move(totals);
    r["stages"] = std::move(stages);
    r["kernels"] = std::move(kernels);  // per kernel name: the duration of every launch, all steps
    r["launches"] = double(dev::launch_count() - launches0 - flushes);
    r["pixels"] = double(ts.negative ? ts.negative.pixels() : ts.source.pixels());
    return json::write(r);
}

}  // namespace spkb

using namespace spkb;

extern "C" {

SPK_API spk_engine* spk_engine_create(const char* resources_dir, void* device) {
    return create(resources_dir, device, SPK_DEVICE_DESKTOP);
}

SPK_API spk_engine* spk_engine_create_for_device(const char* resources_dir, void* device, int32_t device_type) {
    return create(resources_dir, device, device_type);
}

SPK_API void spk_engine_destroy(spk_engine* engine) {
    last_error::clear();
    if (!engine) return;
    Engine* e = E(engine);
    std::set<Session*> ss;
    {
        std::lock_guard<std::mutex> g(e->m);
        ss.swap(e->sessions);
    }
    DeviceGuard dg(e->device);
    for (Session* s : ss) delete s;
    delete e;
}

SPK_API size_t spk_engine_trim(spk_engine* engine) {
    last_error::clear();
    if (!engine) return 0;
    size_t freed = 0;
    try {
        Engine* e = E(engine);
        DeviceGuard dg(e->device);
        std::lock_guard<std::mutex> g(e->m);
        for (Session* s : e->sessions) cudaStreamSynchronize(s->stream);
        freed += device_pool_trim(e->device);
        freed += output_trim();
    } catch (...) {
        map_exception();
    }
    return freed;
}

SPK_API const char* spk_build_info(void) {
    static const std::string s = build_info_string();
    return s.c_str();
}

SPK_API const char* spk_capabilities(spk_engine* engine) {
    if (!engine) return "";
    Engine* e = E(engine);
    std::lock_guard<std::mutex> g(e->m);
    json::Value c;
    c["engine"] = SPK_ENGINE_NAME;
    c["version"] = SPK_VERSION_STRING;
    c["transport_version"] = SPK_TRANSPORT_VERSION;
    c["schema_version"] = SPK_SCHEMA_VERSION;
    c["backend"] = "cuda sm_100a";
    c["device"] = e->device;
    c["effect_versions"] =
        "halation=reference;grain=reference;glare=absent;print_spatial=reference;dir_couplers=reference";
    e->capabilities = json::write(c);
    return e->capabilities.c_str();
}

SPK_API const char* spk_params_schema(spk_engine* engine) { return engine ? schema_json().c_str() : ""; }

// The memory report in the reference's shape (src/session/engine.cpp:246-319): {total_bytes, pool,
// persistent, pressure}. Here "pool" is the per-frame scratch of CUDA's stream-ordered device pool, and
// "persistent" what outlives a render: the cudaMalloc'd tables (the engine's cached pipelines, output
// images excluded) plus each session's frame, tier images and cached negatives, which live in the same
// device pool but are held from render to render. total_bytes = pool.total_bytes + persistent.bytes. The
// stream-ordered pool reuses freed memory in stream order, so nothing is pending and its free blocks are
// not counted as buffers; no memory-pressure monitor or idle trim runs on this device.
SPK_API const char* spk_memory_report(spk_engine* engine) {
    if (!engine) return "";
    Engine* e = E(engine);
    std::lock_guard<std::mutex> g(e->m);
    const DeviceMemory dm = device_memory(e->device);
    uint64_t held = 0, held_buffers = 0, src = 0, neg = 0, nneg = 0;
    json::Array per;
    for (Session* s : e->sessions) {
        uint64_t s_src = s->source ? s->source.bytes() : 0, s_neg = 0, s_n = 0, s_held = s_src;
        held_buffers += s->source ? 1 : 0;
        for (const TierState& t : s->tiers) {
            if (t.negative) {
                s_neg += t.negative.bytes();
                ++s_n;
                ++held_buffers;
            }
            if (t.source && t.source.data() != s->source.data()) {
                s_held += t.source.bytes();
                ++held_buffers;
            }
        }
        if (s->meter_image && s->meter_image.data() != s->tiers[int(Tier::Live)].source.data()) {
            s_held += s->meter_image.bytes();
            ++held_buffers;
        }
        s_held += s_neg;
        json::Value r;
        r["session_id"] = s->id;
        r["source_bytes"] = double(s_src);
        r["cached_negative_bytes"] = double(s_neg);
        r["negatives"] = double(s_n);
        per.push_back(std::move(r));
        src += s_src;
        neg += s_neg;
        nneg += s_n;
        held += s_held;
    }
    auto minus = [](uint64_t a, uint64_t b) { return a > b ? a - b : uint64_t(0); };
    const uint64_t pool_total = minus(dm.reserved, held), pool_live = minus(dm.used, held);
    const uint64_t live_buffers = minus(dm.scratch_live, held_buffers);
    json::Value audit;
    audit["allocations"] = double(dm.scratch_allocations);
    audit["reuses"] = 0.0;  // the device pool's own reuse is not observable
    audit["persistent_allocations"] = double(dm.persistent_allocations);
    audit["reuse_bytes_requested"] = 0.0;
    audit["reuse_bytes_taken"] = 0.0;
    audit["reuse_max_taken"] = 0.0;
    audit["reuse_max_taken_for_request"] = 0.0;
    audit["pending_held"] = 0.0;
    audit["live_underflows"] = 0.0;
    audit["over_releases"] = 0.0;
    audit["reclaim_while_encoding"] = 0.0;
    json::Value pool;
    pool["total_bytes"] = double(pool_total);
    pool["live_bytes"] = double(pool_live);
    pool["free_bytes"] = double(minus(dm.reserved, dm.used));
    pool["pending_bytes"] = 0.0;
    pool["buffers"] = double(live_buffers);
    pool["live_buffers"] = double(live_buffers);
    pool["free_buffers"] = 0.0;
    pool["pending_buffers"] = 0.0;
    pool["frame_high_water_bytes"] = double(minus(dm.used_high, held));
    pool["audit"] = std::move(audit);
    json::Value pers;
    pers["bytes"] = double(dm.persistent_bytes + held);
    pers["buffers"] = double(dm.persistent_live + held_buffers);
    pers["file_backed_bytes"] = 0.0;
    pers["file_backed_buffers"] = 0.0;
    pers["source_bytes"] = double(src);
    pers["cached_negative_bytes"] = double(neg);
    pers["negatives"] = double(nneg);
    pers["sessions"] = std::move(per);
    json::Value pr;
    pr["monitor"] = false;
    pr["warn_events"] = 0.0;
    pr["critical_events"] = 0.0;
    pr["critical_pending"] = false;
    pr["idle_trim_seconds"] = 0.0;
    pr["idle_trims"] = 0.0;
    json::Value r;
    r["total_bytes"] = double(pool_total + dm.persistent_bytes + held);
    r["pool"] = std::move(pool);
    r["persistent"] = std::move(pers);
    r["pressure"] = std::move(pr);
    e->memory_report = json::write(r);
    return e->memory_report.c_str();
}

// Warm-up (reference src/session/engine.cpp:331-412): load two profiles, build a private set-up, develop
// and print a 64 x 64 frame of 0.18 told it is a 1600 px frame, on a private stream and seed sequence.
// A failing step is reported in the reply and ends the sequence.
SPK_API spk_status spk_warm_up(spk_engine* engine, const char* film_stock, const char* print_stock, char** out_json) {
    last_error::clear();
    if (!engine) return invalid("engine is NULL");
    return guarded([&] {
        Engine& e = *E(engine);
        using clock = std::chrono::steady_clock;
        auto ms_since = [](clock::time_point t0) {
            return std::chrono::duration<double, std::milli>(clock::now() - t0).count();
        };
        auto r2 = [](double ms) { return std::round(ms * 100.0) / 100.0; };
        const std::string film_id = film_stock && *film_stock ? film_stock : "kodak_portra_400";
        const std::string print_id = print_stock && *print_stock ? print_stock : "kodak_portra_endura";
        const clock::time_point t_all = clock::now();
        json::Array steps;
        auto run_step = [&](const char* name, auto&& fn) -> bool {
            const clock::time_point t0 = clock::now();
            json::Value st;
            st["name"] = name;
            bool ok = true;
            try {
                fn();
            } catch (const std::exception& ex) {
                ok = false;
                st["error"] = std::string(ex.what());
            }
            st["ok"] = ok;
            st["ms"] = r2(ms_since(t0));
            steps.push_back(std::move(st));
            return ok;
        };
        DeviceGuard dg(e.device);
        ParamSet p;
        p.set(P::film_stock, film_id);
        p.set(P::print_stock, print_id);
        std::shared_ptr<const Profile> fp, pp;
        Pipeline pl;
        cudaStream_t stream = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "warm-up stream");
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
        } sg{stream};
        Pool pool(stream);
        bool ok = run_step("profiles", [&] {
            fp = e.res->profile(film_id);
            pp = e.res->profile(print_id);
            if (auto pack = e.res->neutral_filters(print_id, p.s(P::enlarger_illuminant), *fp)) {
                p.set(P::c_filter_neutral, (*pack)[0]);
                p.set(P::m_filter_neutral, (*pack)[1]);
                p.set(P::y_filter_neutral, (*pack)[2]);
            }
        });
        if (ok)
            ok = run_step("pipeline", [&] {
                check_supported(p);
                auto fs = build_film_setup(p, fp, *e.res);
                pl.print = build_print_setup(p, *fs, pp, *e.res, e.cam16, true);
                pl.film = fs;
                upload_tables(pool, stream, pl);
            });
        if (ok)
            run_step("kernels", [&] {
                constexpr uint32_t kSide = 64;
                Plane src = make_plane(pool, kSide, kSide);
                const std::vector<float> grey(size_t(kSide) * kSide * 3, 0.18f);
                cuda_check(cudaMemcpyAsync(src.data(), grey.data(), src.bytes(), cudaMemcpyHostToDevice, stream),
                           "warm-up frame");
                RenderCtx ctx{pool, stream};
                ctx.rho_tier = 1.0;
                ctx.pitch_um = 1000.0 * p.f(P::film_format_mm) / double(kMeterLongEdge);
                SeedSequence seeds;  // private: never a session's
                const uint32_t film_seed = p.b(P::grain_active) ? seeds.next() : kNoGrainFilmSeed;
                Plane neg = develop(ctx, pl, src, film_seed, std::nullopt);
                ctx.print_seed = pl.print->glare_draws() ? seeds.next() : 0u;
                OutputImage* img = output_acquire(e.device, kSide, kSide);
                try {
                    print_scan_encode(ctx, pl, LiveParams::from(p), neg, img);
                    cuda_check(cudaStreamSynchronize(stream), "warm-up");
                } catch (...) {
                    output_release(img);
                    throw;
                }
                output_release(img);
            });
        json::Value r;
        r["already_warm"] = false;
        r["film_stock"] = film_id;
        r["print_stock"] = print_id;
        r["render_core"] = "native-cuda";
        r["steps"] = std::move(steps);
        r["total_ms"] = r2(ms_since(t_all));
        put_json(out_json, json::write(r));
        return SPK_OK;
    });
}

SPK_API spk_session* spk_open(spk_engine* engine, const spk_image* input, const char* delta, char** out_json) {
    last_error::clear();
    if (!engine) {
        invalid("engine is NULL");
        return nullptr;
    }
    if (!input) {
        invalid("input is NULL");
        return nullptr;
    }
    try {
        std::string reply;
        Session* s = open_session(*E(engine), input->data, false, input->width, input->height, input->channels, delta,
                                  out_json ? &reply : nullptr);
        put_json(out_json, reply);
        return reinterpret_cast<spk_session*>(s);
    } catch (...) {
        map_exception();
        return nullptr;
    }
}

SPK_API spk_session* spk_open_device(spk_engine* engine, const spk_device_image* input, const char* delta,
                                     char** out_json) {
    last_error::clear();
    if (!engine) {
        invalid("engine is NULL");
        return nullptr;
    }
    if (!input) {
        invalid("input is NULL");
        return nullptr;
    }
    try {
        std::string reply;
        Session* s = open_session(*E(engine), input->buffer, true, input->width, input->height, input->channels, delta,
                                  out_json ? &reply : nullptr);
        put_json(out_json, reply);
        return reinterpret_cast<spk_session*>(s);
    } catch (...) {
        map_exception();
        return nullptr;
    }
}

SPK_API spk_status spk_set_params(spk_session* session, const char* delta_text, char** out_json) {
    last_error::clear();
    if (!session) return invalid("session is NULL");
    return guarded([&] {
        Session& s = *S(session);
        const Delta d = validate_delta(delta_text ? delta_text : "", DeltaContext::SetParams);
        std::lock_guard<std::mutex> lock(s.m);
        DeviceGuard dg(s.engine->device);
        ParamSet cand = s.params;
        apply_delta(cand, d);
        auto film = s.film, print = s.print;
        if (d.has_stock) {
            film = s.engine->res->profile(cand.s(P::film_stock));
            print = s.engine->res->profile(cand.s(P::print_stock));
            s.digest(cand, *film);
        }
        if (d.any_rebuild) {
            Pipeline pl = s.build(cand, film, print);
            s.pipe = std::move(pl);
            s.seeds = SeedSequence{};
        }
        s.live = LiveParams::from(cand);
        const uint32_t old_live = uint32_t(s.params.i(P::preview_long_edge));
        // a change to a field of the meter's key re-arms the meter (reference src/session/session.cpp:34-36)
        constexpr P kMeterKey[] = {P::input_color_space,    P::input_cctf_decoding, P::geometry_crop_x,
                                   P::geometry_crop_y,      P::geometry_crop_w,     P::geometry_crop_h,
                                   P::geometry_rotation_deg, P::geometry_quarter_turns, P::geometry_flip_h,
                                   P::geometry_flip_v};
        for (P k : kMeterKey)
            if (json::write(s.params.get(size_t(k))) != json::write(cand.get(size_t(k)))) s.meter.reset();
        s.params = cand;
        s.film = film;
        s.print = print;
        if (d.any_shoot)
            for (TierState& t : s.tiers) t.negative = Plane{};
        // a new preview_long_edge that changes the live tier's size drops the live tier's image and negative
        // (reference src/session/session.cpp:247-251)
        if (d.has_preview_long_edge) {
            const Size2 a = downscale_size(s.source.w, s.source.h, old_live);
            const Size2 b = downscale_size(s.source.w, s.source.h, uint32_t(s.params.i(P::preview_long_edge)));
            if (a.w != b.w || a.h != b.h) s.tiers[int(Tier::Live)] = TierState{};
        }
        json::Value r;
        r["invalidated"] = d.any_shoot ? "shoot" : "print";
        r["params"] = s.params.to_json();
        put_json(out_json, json::write(r));
        return SPK_OK;
    });
}

SPK_API spk_status spk_get_params(spk_session* session, char** out_json) {
    if (!session) return invalid("session is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        put_json(out_json, json::write(s.params.to_json()));
        return SPK_OK;
    });
}

SPK_API void spk_session_release(spk_session* session) {
    last_error::clear();
    if (!session) return;
    Session* s = S(session);
    Engine* e = s->engine;
    {
        std::lock_guard<std::mutex> g(e->m);
        e->sessions.erase(s);
    }
    DeviceGuard dg(e->device);
    cudaStreamSynchronize(s->stream);
    delete s;
}

SPK_API spk_status spk_render(spk_session* session, const char* tier, spk_result* out) {
    return render_common(session, tier, out, false);
}

SPK_API spk_status spk_reprint(spk_session* session, const char* tier, spk_result* out) {
    return render_common(session, tier, out, true);
}

SPK_API void spk_result_free(spk_result* result) {
    last_error::clear();
    if (!result || !result->texture) return;
    output_release(static_cast<OutputImage*>(result->texture));
    result->texture = nullptr;
    result->rgba16 = nullptr;
}

// The solver (reference src/session/session.cpp:450-499): never changes parameters. exposure: the meter
// (metered now, or the kept one) gives the session method's EV and the four intent EVs; filter_pack: the
// neutral filter database's row for (paper, enlarger illuminant, film), else the current values.
SPK_API spk_status spk_solve(spk_session* session, const char* target_in, char** out_json) {
    last_error::clear();
    if (!session) return invalid("session is NULL");
    return guarded([&] {
        Session& s = *S(session);
        const std::string target = target_in && *target_in ? target_in : "both";
        std::lock_guard<std::mutex> lock(s.m);
        const bool exposure = target == "exposure" || target == "both";
        const bool pack = target == "filter_pack" || target == "both";
        if (!exposure && !pack) fail_user("unknown solve target '" + target + "'; expected exposure, filter_pack or both");
        json::Value solved = json::Object{};
        json::Value r;
        if (exposure) {
            DeviceGuard dg(s.engine->device);
            const MeterValues* m = nullptr;
            try {
                m = &s.ensure_meter();
            } catch (const Error& e) {
                fail_gpu(e.what());  // the meter failed: a render failure
            }
            solved["exposure_compensation_ev"] = m->ev(s.params.s(P::auto_exposure_method));
            json::Value by;
            by["balanced"] = m->balanced;
            by["center"] = m->center;
            by["protect_highlights"] = m->protect_highlights;
            by["protect_shadows"] = m->protect_shadows;
            r["exposure_ev_by_method"] = std::move(by);
        }
        if (pack) {
            Vec3 v{s.params.f(P::c_filter_neutral), s.params.f(P::m_filter_neutral), s.params.f(P::y_filter_neutral)};
            try {
                if (auto hit = s.engine->res->neutral_filters(s.params.s(P::print_stock),
                                                              s.params.s(P::enlarger_illuminant), *s.film))
                    v = *hit;
            } catch (const std::exception& e) {
                fail_internal(std::string("filter resolution failed: ") + e.what());
            }
            solved["c_filter_neutral"] = v[0];
            solved["m_filter_neutral"] = v[1];
            solved["y_filter_neutral"] = v[2];
        }
        r["solved_params"] = std::move(solved);
        put_json(out_json, json::write(r));
        return SPK_OK;
    });
}

SPK_API const char* spk_print_lut_catalog(spk_engine* engine) {
    return engine ? E(engine)->res->print_lut_catalog().c_str() : "{}";
}

SPK_API spk_status spk_print_lut_table(spk_engine* engine, const char* print_stock, const float** out_table,
                                       uint32_t* out_size) {
    last_error::clear();
    if (!engine || !print_stock || !out_table || !out_size) return invalid("a required pointer is NULL");
    return guarded([&] {
        // the table lives in the engine's resources for the engine's life
        const std::shared_ptr<const PrintLut> t = E(engine)->res->print_lut(print_stock);
        *out_table = t->table.data();
        *out_size = t->size;
        return SPK_OK;
    });
}

SPK_API spk_status spk_preview_stock_lut(spk_session* session, const char* print_stock, const char* tier,
                                         spk_result* out, char** out_json) {
    last_error::clear();
    if (!session || !out) return invalid("a required pointer is NULL");
    std::memset(out, 0, sizeof *out);
    return guarded([&] {
        preview_stock_lut(*S(session), print_stock, tier, out, out_json);
        return SPK_OK;
    });
}

namespace {
// gamut_compress_json (reference src/print/cam16.cpp:246-277): keys optional; not an object is
// SPK_ERR_INVALID_ARG, an unknown algorithm SPK_ERR_USER; an array that is not three numbers is ignored
struct GamutOptions {
    std::string algorithm = "cam16ucs";
    std::array<double, 3> knee{0.0, 1.0, 6.0}, lc{0.7, 1.0, 2.2};
    bool lc_active = true;
};
GamutOptions parse_gamut(const char* text) {
    GamutOptions g;
    if (!text || !*text) return g;
    json::Value v;
    try {
        v = json::parse(text);
    } catch (const json::ParseError& e) {
        fail_invalid(std::string("gamut_compress_json: ") + e.what());
    }
    if (!v.is_object()) fail_invalid("gamut_compress_json must be a JSON object");
    if (const json::Value* a = v.find("algorithm")) {
        if (!a->is_string() || (a->as_string() != "cam16ucs" && a->as_string() != "off"))
            fail_user("unknown gamut compression algorithm" + (a->is_string() ? " '" + a->as_string() + "'" : std::string()) +
                      " (expected cam16ucs or off)");
        g.algorithm = a->as_string();
    }
    auto triple = [&](const char* key, std::array<double, 3>& out) {
        const json::Value* a = v.find(key);
        if (!a || !a->is_array() || a->as_array().size() != 3) return;
        std::array<double, 3> t{};
        for (size_t i = 0; i < 3; ++i) {
            if (!a->as_array()[i].is_number()) return;
            t[i] = a->as_array()[i].as_number();
        }
        out = t;
    };
    triple("knee", g.knee);
    triple("lightness_compression", g.lc);
    if (const json::Value* b = v.find("lightness_compression_active"); b && b->is_bool()) g.lc_active = b->as_bool();
    return g;
}
}  // namespace

// The output transform (reference src/print/cam16.cpp:306-347): a fetch, never a render. The matrix is
// XYZ -> RGB(dst) . CAT02(white src -> white dst, when the whites differ) . RGB -> XYZ(src); the gamut
// constants and the C_max table are those of dst, the table engine-owned for the engine's life.
SPK_API spk_status spk_output_transform(spk_engine* engine, const char* src, const char* dst, const char* gamut_json,
                                        char** out_json, const float** out_cmax, uint32_t* out_cmax_count) {
    last_error::clear();
    if (!engine) return invalid("engine is NULL");
    if (!src) return invalid("src_cs is NULL");
    if (!dst) return invalid("dst_cs is NULL");
    if (!out_json || !out_cmax || !out_cmax_count) return invalid("a required output pointer is NULL");
    return guarded([&] {
        Engine& e = *E(engine);
        const GamutOptions g = parse_gamut(gamut_json);
        auto space = [&](const char* name) {
            if (!cctf_of(name)) fail_user("unknown colour space '" + std::string(name) + "'");
            auto cs = colour_space(e.res->blob(), name);
            if (!cs) fail_user("colour space '" + std::string(name) + "' has no baked matrices or whitepoint");
            if (cs->whitepoint[1] == 0.0) fail_user("colour space '" + std::string(name) + "' has a whitepoint with y = 0");
            return *cs;
        };
        const ColourSpace sc = space(src), dc = space(dst);
        auto cat02 = cat_matrix(e.res->blob(), "CAT02");
        if (!cat02) fail_user("the constants blob has no colour/cat/CAT02");
        Mat3 m = dc.xyz_to_rgb;
        if (auto a = von_kries(sc.whitepoint, dc.whitepoint, *cat02, Guard::Target)) m = mat3_mul(m, *a);
        m = mat3_mul(m, sc.rgb_to_xyz);
        const std::shared_ptr<const Cam16Tables> t = e.cam16.get(*e.res, dst);
        const Cam16Constants& c = t->k;
        auto mat = [](const Mat3& v) {
            json::Array a;
            for (double x : v) a.emplace_back(x);
            return json::Value(std::move(a));
        };
        json::Value gc;
        gc["algorithm"] = g.algorithm;
        gc["m_to_xyz"] = mat(t->m_to_xyz);
        gc["m_to_rgb"] = mat(t->m_to_rgb);
        const double k[22] = {c.F_L, c.N_bb, c.N_cb, c.n, c.z, c.A_w, c.c, c.N_c, 1.0, 110.0, -M_PI,
                              2.0 * M_PI / 720.0, g.knee[0], g.knee[1], g.knee[2], g.lc_active ? g.lc[0] : 0.0,
                              g.lc_active ? g.lc[1] : 1.0, g.lc_active ? g.lc[2] : 1.0, c.J_white, c.D_rgb[0],
                              c.D_rgb[1], c.D_rgb[2]};
        json::Array ka;
        for (double v : k) ka.emplace_back(v);
        gc["k"] = json::Value(std::move(ka));
        gc["cmax_rows"] = 64;
        gc["cmax_cols"] = 720;
        gc["lightness_compression_active"] = g.lc_active;
        json::Value r;
        r["source_color_space"] = sc.name;
        r["target_color_space"] = dc.name;
        r["source_cctf_mode"] = int(sc.cctf);
        r["target_cctf_mode"] = int(dc.cctf);
        r["matrix"] = mat(m);
        r["gamut_compress"] = std::move(gc);
        put_json(out_json, json::write(r));
        *out_cmax = t->cmax32.data();
        *out_cmax_count = uint32_t(t->cmax32.size());
        return SPK_OK;
    });
}

SPK_API void spk_cancel(spk_session* session, const char* progress_id) {
    if (!session) return;
    S(session)->progress.cancel(progress_id);
}

SPK_API spk_status spk_progress(spk_session* session, const char* progress_id, char** out_json) {
    if (!session) return invalid("session is NULL");
    return guarded([&] {
        const json::Value r = S(session)->progress.snapshot(progress_id);
        put_json(out_json, json::write(r));
        return SPK_OK;
    });
}

SPK_API void spk_string_free(char* s) { std::free(s); }

SPK_API const char* spk_last_error(spk_engine*) { return last_error::get(); }

// ---- extensions -----------------------------------------------------------------------------------

SPK_API spk_status spkx_session_set_halation(spk_session* session, uint32_t n, const double* weights,
                                             const double* sigmas, const double* strength) {
    last_error::clear();
    if (!session) return invalid("session is NULL");
    if (n > SPKB_MAX_COMPONENTS) return invalid("at most 8 halation components");
    if (n > 0 && (!weights || !sigmas || !strength)) return invalid("a required array is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        if (n == 0) {
            s.hal.reset();
        } else {
            HalationOverride o;
            for (uint32_t k = 0; k < n; ++k) {
                MixtureComponent m;
                for (int c = 0; c < 3; ++c) {
                    m.weight[c] = weights[3 * k + c];
                    m.sigma[c] = sigmas[3 * k + c];
                }
                o.comps.push_back(m);
            }
            for (int c = 0; c < 3; ++c) o.strength[c] = strength[c];
            s.hal = o;
        }
        for (TierState& t : s.tiers) t.negative = Plane{};
        return SPK_OK;
    });
}

SPK_API spk_status spkx_session_profile(spk_session* session, const char* tier, int32_t reprint, uint32_t steps,
                                        char** out_json) {
    last_error::clear();
    if (!session) return invalid("session is NULL");
    return guarded([&] {
        put_json(out_json, session_profile(*S(session), tier, reprint != 0, steps));
        return SPK_OK;
    });
}

SPK_API spk_status spkx_session_meter(spk_session* session, char** out_json) {
    last_error::clear();
    if (!session || !out_json) return invalid("a required pointer is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        DeviceGuard dg(s.engine->device);
        if (!s.params.b(P::auto_exposure)) fail_user("auto_exposure is off in this session");
        const MeterValues& m = s.ensure_meter();
        json::Value r;
        r["center_weighted"] = m.center_weighted;
        r["average"] = m.average;
        r["median"] = m.median;
        r["balanced"] = m.balanced;
        r["center"] = m.center;
        r["protect_highlights"] = m.protect_highlights;
        r["protect_shadows"] = m.protect_shadows;
        put_json(out_json, json::write(r));
        return SPK_OK;
    });
}

SPK_API spk_status spkx_session_tier_image(spk_session* session, const char* tier, float* out, size_t capacity,
                                          uint32_t* width, uint32_t* height) {
    last_error::clear();
    if (!session || !width || !height) return invalid("a required pointer is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        auto t = parse_tier(tier);
        if (!t) fail_invalid("unknown tier");
        DeviceGuard dg(s.engine->device);
        const TierState& ts = s.tier_source(*t);
        *width = ts.source.w;
        *height = ts.source.h;
        if (out) {
            if (capacity < 3 * ts.source.pixels()) fail_invalid("output capacity too small");
            cuda_check(cudaMemcpyAsync(out, ts.source.data(), ts.source.bytes(), cudaMemcpyDeviceToHost, s.stream),
                       "tier image copy");
            cuda_check(cudaStreamSynchronize(s.stream), "tier image copy");
        }
        return SPK_OK;
    });
}

SPK_API spk_status spkx_session_negative(spk_session* session, const char* tier, float* out, size_t capacity) {
    last_error::clear();
    if (!session || !out) return invalid("a required pointer is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        auto t = parse_tier(tier);
        if (!t) fail_invalid("unknown tier");
        const TierState& ts = s.tiers[int(*t)];
        if (!ts.negative) fail_user("no cached negative for this tier");
        if (capacity < 3 * ts.negative.pixels()) fail_invalid("output capacity too small");
        DeviceGuard dg(s.engine->device);
        cuda_check(cudaMemcpyAsync(out, ts.negative.data(), ts.negative.bytes(), cudaMemcpyDeviceToHost, s.stream),
                   "negative copy");
        cuda_check(cudaStreamSynchronize(s.stream), "negative copy");
        return SPK_OK;
    });
}

SPK_API spk_status spkx_session_set_print_mode(spk_session* session, const char* mode, uint32_t bins) {
    last_error::clear();
    if (!session || !mode) return invalid("a required pointer is NULL");
    const std::string m(mode);
    int code = -2;
    if (m == "fp32") code = -1;
    if (m == "fp32_generic") code = SPKB_SPEC_F32;
    if (m == "fp64") code = SPKB_SPEC_F64;
    if (m == "tf32") code = SPKB_SPEC_TF32;
    if (m == "bf16") code = SPKB_SPEC_BF16;
    if (m == "bf16x3") code = SPKB_SPEC_BF16X3;
    if (code == -2) return invalid("print mode must be fp32, fp32_generic, fp64, tf32, bf16 or bf16x3");
    if (bins != SPKB_NL && bins != 401) return invalid("print wavelengths must be 81 or 401");
    if (code == -1 && bins != SPKB_NL) code = SPKB_SPEC_F32;  // the binary32 print kernel holds 81 wavelengths
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        s.print_mode = code;
        s.print_bins = bins;
        return SPK_OK;
    });
}

SPK_API spk_status spkx_print_negative(spk_session* session, const float* negative, uint32_t width, uint32_t height,
                                       uint16_t* rgba16, uint32_t row_stride_px, float* contraction, double* print_ms) {
    last_error::clear();
    if (!session || !negative || !rgba16) return invalid("a required pointer is NULL");
    if (width == 0 || height == 0 || uint64_t(width) * height > kMaxPixels) return invalid("frame size out of range");
    if (row_stride_px < width) return invalid("row_stride_px is below the width");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        if (contraction && s.print_mode < 0)
            fail_invalid("the enlarger integral is written by the spectral-mode print kernel only");
        DeviceGuard dg(s.engine->device);
        Plane neg = make_plane(s.pool, width, height);
        cuda_check(cudaMemcpyAsync(neg.data(), negative, neg.bytes(), cudaMemcpyDeviceToDevice, s.stream), "negative");
        OutputImage img{};
        img.dev = rgba16;
        img.width = width;
        img.height = height;
        img.stride_px = row_stride_px;
        img.device = s.engine->device;
        RenderCtx ctx{s.pool, s.stream};
        ctx.print_mode = s.print_mode;
        ctx.print_bins = s.print_bins;
        ctx.contraction_out = contraction;
        Timer timer;
        struct HookGuard {
            ~HookGuard() { dev::set_launch_hook(nullptr); }
        } hook_guard;
        if (print_ms) {
            ctx.timer = &timer;
            dev::set_launch_hook(&timer);
        }
        print_scan_encode(ctx, s.pipe, s.live, neg, &img);
        cuda_check(cudaStreamSynchronize(s.stream), "print");
        cuda_check(cudaGetLastError(), "print");
        if (print_ms) {
            *print_ms = 0.0;
            for (const Timer::Mark& k : timer.kernels) {
                const std::string name(k.name);
                if (name != "print" && name != "print_spectral") continue;
                float ms = 0.0f;
                cuda_check(cudaEventElapsedTime(&ms, k.a, k.b), "print timing");
                *print_ms += ms;
            }
        }
        return SPK_OK;
    });
}

SPK_API spk_status spkx_engine_batch_plan(spk_engine* engine, const char* plan) {
    last_error::clear();
    if (!engine) return invalid("engine is NULL");
    const std::string p = plan ? plan : "";
    if (!p.empty() && !valid_plan(p))
        return invalid("batch plan must be \"frames:K\" (K 1..16) or \"persistent:S:C[:G]\" (S even, 2..1048576; "
                       "C 1..65535; G 1..1024)");
    return guarded([&] {
        Engine& e = *E(engine);
        std::lock_guard<std::mutex> g(e.batch_m);
        e.pinned_plan = p;
        return SPK_OK;
    });
}

// Batched renders: this build's extension (no reference counterpart; spk_render per session is the
// reference's only entry, src/abi/abi.cpp:293-308, and every result here is the one spk_render gives).
SPK_API spk_status spkx_render_batch(spk_session* const* sessions, uint32_t n, const char* tier, int32_t reprint,
                                     spk_result* results, char** out_json) {
    last_error::clear();
    if (out_json) *out_json = nullptr;
    if (!sessions) return invalid("sessions is NULL");
    if (!results) return invalid("results is NULL");
    if (n == 0) return invalid("a batch needs at least one session");
    std::memset(results, 0, sizeof(spk_result) * n);
    const int32_t st = guarded([&] {
        std::vector<Session*> ss(n);
        for (uint32_t i = 0; i < n; ++i) ss[i] = S(sessions[i]);
        std::string info;
        render_batch(ss, tier, reprint != 0, results, &info);
        put_json(out_json, info);
        return SPK_OK;
    });
    if (st != SPK_OK)
        for (uint32_t i = 0; i < n; ++i) release_result(&results[i]);
    return st;
}

}  // extern "C"

namespace spkb {

// The same constants before narrowing (binary64), which feed the float64 oracle.
json::Value setup_f64(const FilmSetup& f, const PrintSetup& p, const PrintRun& run, const LiveParams& live,
                      double pitch_um) {
    auto arr = [](const double* v, size_t n) {
        json::Array a;
        for (size_t i = 0; i < n; ++i) a.push_back(json::Value(v[i]));
        return json::Value(std::move(a));
    };
    const Profile& film = *f.profile;
    const size_t K = film.K();
    const double gamma = f.params.f(P::density_curve_gamma);
    std::vector<double> cx(K), cinv(K, 0.0), cy(3 * K);
    for (size_t k = 0; k < K; ++k) {
        cx[k] = film.log_exposure[k] / gamma;
        if (k + 1 < K) {
            const double d = film.log_exposure[k + 1] / gamma - film.log_exposure[k] / gamma;
            cinv[k] = d == 0.0 ? 0.0 : 1.0 / d;
        }
        for (size_t c = 0; c < 3; ++c) cy[c * K + k] = film.normalized(k, c);
    }
    json::Value r;
    r["input_matrix"] = arr(f.input_matrix.data(), 9);
    r["input_cctf_mode"] = int(f.input_space.cctf);
    r["input_rgb_to_xyz"] = arr(f.input_space.rgb_to_xyz.data(), 9);
    r["boost_ev"] = f.params.f(P::halation_boost_ev);
    {
        json::Value ed;
        ed["active"] = p.edr && !p.scanned;
        ed["r_y"] = arr(p.out_cs.rgb_to_xyz.data() + 3, 3);
        ed["lo"] = p.edr_lo;
        ed["hi"] = p.edr_hi;
        ed["toe"] = p.edr_toe;
        ed["shoulder"] = p.edr_shoulder;
        std::vector<double> t;
        if (p.edr) t = p.paper->edr->target;
        ed["table"] = arr(t.data(), t.size());
        r["edr"] = std::move(ed);
    }
    {
        json::Value lv;
        lv["active"] = run.levels;
        lv["m"] = run.m;
        lv["q"] = run.q;
        r["levels"] = std::move(lv);
    }
    r["headroom_ev"] = headroom_applies(f.halation) ? f.halation.headroom_ev : 0.0;
    {
        // the print glare: its binary32 lognormal parameters, the blur at the full tier, the tint
        const PrintSetup& ps = p;
        const double pp = ps.glare_percent * ps.glare_amount;
        json::Value g;
        g["draws"] = !ps.scanned && ps.glare_draws();
        g["mean"] = double(f32(pp));
        g["sd"] = double(f32(ps.glare_roughness * pp));
        g["sigma_full"] = ps.glare_blur_full * std::sqrt(std::max(ps.glare_amount, 0.0));
        g["tint"] = arr(ps.glare_tint.data(), 3);
        r["glare"] = std::move(g);
    }
    r["gain"] = std::pow(2.0, f.params.f(P::exposure_compensation_ev));
    r["table"] = arr(f.table64.data(), f.table64.size());
    r["curve_x"] = arr(cx.data(), K);
    r["curve_inv"] = arr(cinv.data(), K);
    r["curve_y"] = arr(cy.data(), 3 * K);
    {
        // DIR couplers: the matrix, D_max, the pre-inverted curve and the diffusion mixture at this pitch
        json::Value cp;
        cp["active"] = f.couplers;
        cp["m"] = arr(f.coupler_m.data(), 9);
        cp["dmax"] = arr(f.dmax.data(), 3);
        cp["y0"] = arr(f.cy0_64.data(), f.cy0_64.size());
        json::Array dir;
        for (const MixtureComponent& m : dir_diffusion_components(pitch_um)) {
            json::Array pair;
            pair.push_back(arr(m.weight.data(), 3));
            pair.push_back(arr(m.sigma.data(), 3));
            dir.push_back(json::Value(std::move(pair)));
        }
        cp["dir"] = json::Value(std::move(dir));
        r["couplers"] = std::move(cp);
    }
    if (f.grain && f.grain->K) {
        const GrainSetup& g = *f.grain;
        const GrainConstants kc = grain_constants(g, pitch_um);
        double cnt[9], sat[9], dml[9];
        for (int l = 0; l < 3; ++l)
            for (int c = 0; c < 3; ++c) {
                cnt[3 * l + c] = kc.count[l][c];
                sat[3 * l + c] = kc.sat_d[l][c];
                dml[3 * l + c] = kc.dmin_l[l][c];
            }
        r["grain_count"] = arr(cnt, 9);
        r["grain_sat_d"] = arr(sat, 9);
        r["grain_dmin_l"] = arr(dml, 9);
        r["grain_final_blur"] = kc.final_blur;
        std::vector<double> ax(K * 3), gi(K * 3, 0.0);
        for (size_t k = 0; k < K; ++k)
            for (size_t c = 0; c < 3; ++c) ax[k * 3 + c] = g.positive ? -film.normalized(k, c) : film.normalized(k, c);
        for (size_t k = 0; k + 1 < K; ++k)
            for (size_t c = 0; c < 3; ++c) {
                const double st = ax[(k + 1) * 3 + c] - ax[k * 3 + c];
                gi[k * 3 + c] = st == 0.0 ? 0.0 : 1.0 / st;
            }
        r["grain_axis"] = arr(ax.data(), ax.size());
        r["grain_inv"] = arr(gi.data(), gi.size());
        r["grain_layers"] = arr(film.layers.data(), film.layers.size());
    }
    {
        const HalationPlan pl = halation_plan(f.halation, pitch_um);
        auto comps = [&](const std::vector<MixtureComponent>& v) {
            json::Array a;
            for (const MixtureComponent& m : v)
                a.push_back(json::Array{arr(m.weight.data(), 3), arr(m.sigma.data(), 3)});
            return json::Value(std::move(a));
        };
        json::Value hv;
        hv["scatter"] = comps(pl.scatter ? pl.scatter_comps : std::vector<MixtureComponent>{});
        hv["scatter_a"] = arr(pl.scatter_a.data(), 3);
        hv["scatter_b"] = arr(pl.scatter_b.data(), 3);
        hv["bounce"] = comps(pl.bounce ? pl.bounce_comps : std::vector<MixtureComponent>{});
        hv["mix_a"] = arr(pl.mix_a.data(), 3);
        hv["mix_b"] = arr(pl.mix_b.data(), 3);
        r["halation"] = std::move(hv);
        r["lens_blur_px"] = f.params.f(P::lens_blur_um) / pitch_um;
        r["grain_active"] = f.grain && f.grain->active && f.grain->amount > 0.0;
        r["grain_amount"] = f.grain ? f.grain->amount : 0.0;
        r["positive"] = f.positive;
    }
    r["enl_eps"] = arr(run.eps_n.data(), 243);
    r["enl_beta"] = arr(run.beta_n.data(), 81);
    r["enl_wt"] = arr(run.w_n.data(), 243);
    r["enl_g"] = arr(run.g.data(), 3);
    r["enl_o"] = arr(run.o.data(), 3);
    r["k_gain"] = live.print_exposure * run.kappa_bw;  // the levels' exposure correction included
    r["scan_eps"] = arr(p.scan_eps.data(), 243);
    r["scan_beta"] = arr(p.scan_beta.data(), 81);
    r["scan_wt"] = arr(p.scan_wt.data(), 243);
    if (p.paper) {
        const Profile& paper = *p.paper;
        const size_t pk = paper.K();
        std::vector<double> pr(pk, 0.0);
        for (size_t i = 0; i + 1 < pk; ++i) {
            const double d = paper.log_exposure[i + 1] - paper.log_exposure[i];
            pr[i] = d == 0.0 ? 0.0 : 1.0 / d;
        }
        r["paper_x"] = arr(paper.log_exposure.data(), pk);
        r["paper_r"] = arr(pr.data(), pk);
        r["paper_y"] = arr(p.paper_y64.data(), p.paper_y64.size());
    }
    r["to_rgb"] = arr(p.to_rgb64.data(), 9);
    r["m_nid"] = arr(p.m_nid64.data(), 9);
    const Cam16Constants& k = p.cam->k;
    const double cam[] = {k.F_L, k.N_bb, k.N_cb, k.n, k.z, k.A_w, k.c, k.N_c, 1.0, 110.0, -M_PI, 2.0 * M_PI / 720.0,
                          0.0, 1.0, 6.0, 0.7, 1.0, 2.2, k.J_white, k.D_rgb[0], k.D_rgb[1], k.D_rgb[2]};
    r["cam_k"] = arr(cam, 22);
    r["cam_m_to_xyz"] = arr(p.cam->m_to_xyz.data(), 9);
    r["cam_m_to_rgb"] = arr(p.cam->m_to_rgb.data(), 9);
    r["cam_m16"] = arr(k.m16.data(), 9);
    static constexpr double kInvPublished[9] = {1.86206786,  -1.01125463, 0.14918677,  0.38752654, 0.62144744,
                                                -0.00897398, -0.01584150, -0.03412294, 1.04996444};
    r["cam_m16_inv"] = arr(kInvPublished, 9);
    r["cmax"] = arr(p.cam->cmax64.data(), p.cam->cmax64.size());
    r["scanner_lens_blur"] = p.scanner_lens_blur_px;
    r["unsharp_sigma"] = p.unsharp_sigma_full;
    r["unsharp_amount"] = p.unsharp_amount;
    r["cctf_active"] = p.cctf;
    r["cctf_mode"] = p.cctf_mode;
    r["printed"] = !p.scanned;
    return r;
}

// The narrowed kernel constants of a pipeline, for set-up parity checks against the reference.
std::string setup_json(const FilmSetup& f, const PrintSetup& p, const LiveParams& live, double pitch_um) {
        auto arr = [](const float* v, size_t n) {
            json::Array a;
            for (size_t i = 0; i < n; ++i) a.push_back(json::Value(double(v[i])));
            return json::Value(std::move(a));
        };
        json::Value r;
        r["input_matrix"] = arr(f.input_matrix_f32.data(), 9);
        r["L"] = f.L;
        r["table"] = arr(f.table32.data(), f.table32.size());
        r["curve_x"] = arr(f.cx.data(), f.cx.size());
        r["curve_inv"] = arr(f.cinv.data(), f.cinv.size());
        r["curve_y"] = arr(f.cy.data(), f.cy.size());
        if (f.grain) {
            const GrainConstants kc = grain_constants(*f.grain, pitch_um);
            float cnt[9], sat[9], dml[9];
            for (int l = 0; l < 3; ++l)
                for (int c = 0; c < 3; ++c) {
                    cnt[3 * l + c] = f32(kc.count[l][c]);
                    sat[3 * l + c] = f32(kc.sat_d[l][c]);
                    dml[3 * l + c] = f32(kc.dmin_l[l][c]);
                }
            r["grain_count"] = arr(cnt, 9);
            r["grain_sat_d"] = arr(sat, 9);
            r["grain_dmin_l"] = arr(dml, 9);
            r["grain_axis"] = arr(f.grain->axis.data(), f.grain->axis.size());
            r["grain_inv"] = arr(f.grain->inv.data(), f.grain->inv.size());
            r["grain_layers"] = arr(f.grain->layers.data(), f.grain->layers.size());
        }
        const PrintRun run = compute_run(p, live);
        r["enl_eps"] = arr(run.enl32.eps, 243);
        r["enl_beta"] = arr(run.enl32.beta, 81);
        r["enl_wt"] = arr(run.enl32.wt, 243);
        float g[3], o[3];
        for (int c = 0; c < 3; ++c) {
            g[c] = f32(run.g[c]);
            o[c] = f32(run.o[c]);
        }
        r["enl_g"] = arr(g, 3);
        r["enl_o"] = arr(o, 3);
        r["k_gain"] = double(run.k_gain);
        r["scan_eps"] = arr(p.scan32.eps, 243);
        r["scan_beta"] = arr(p.scan32.beta, 81);
        r["scan_wt"] = arr(p.scan32.wt, 243);
        r["paper"] = arr(p.paper_tab.data(), p.paper_tab.size());
        r["to_rgb"] = arr(p.to_rgb, 9);
        r["m_nid"] = arr(p.m_nid, 9);
        const Cam16Args& q = p.cam_args;
        const float cam[] = {q.f_l, q.n_bb, q.n_cb, q.n, q.z, q.a_w, q.c, q.n_c, q.j_first, q.j_last, q.h_first,
                             q.h_step, q.knee[0], q.knee[1], q.knee[2], q.lc[0], q.lc[1], q.lc[2], q.j_white,
                             q.d_rgb[0], q.d_rgb[1], q.d_rgb[2]};
        r["cam_k"] = arr(cam, 22);
        r["cam_m_to_xyz"] = arr(q.m_to_xyz, 9);
        r["cam_m_to_rgb"] = arr(q.m_to_rgb, 9);
        r["cmax"] = arr(p.cam->cmax32.data(), p.cam->cmax32.size());
    r["f64"] = setup_f64(f, p, run, live, pitch_um);
    return json::write(r);
}

// Parameters of an open (reference src/session/session.cpp:142-152): defaults, the delta's stocks,
// the digest, the forced working output space, the delta, the digest again.
ParamSet open_params(const Resources& res, const Delta& d, std::shared_ptr<const Profile>& film,
                     std::shared_ptr<const Profile>& print) {
    ParamSet p;
    for (const auto& [fid, v] : d.fields)
        if (fid == size_t(P::film_stock) || fid == size_t(P::print_stock)) p.set(fid, v);
    film = res.profile(p.s(P::film_stock));
    print = res.profile(p.s(P::print_stock));
    auto digest = [&] {
        if (auto pack = res.neutral_filters(p.s(P::print_stock), p.s(P::enlarger_illuminant), *film)) {
            p.set(P::c_filter_neutral, (*pack)[0]);
            p.set(P::m_filter_neutral, (*pack)[1]);
            p.set(P::y_filter_neutral, (*pack)[2]);
        }
    };
    digest();
    p.set(P::output_color_space, "ProPhoto RGB");
    p.set(P::output_cctf_encoding, true);
    apply_delta(p, d);
    digest();
    return p;
}

}  // namespace spkb

extern "C" {

SPK_API spk_status spkx_session_develop_debug(spk_session* session, const char* tier, uint32_t seed, float* negative,
                                              float* counts) {
    last_error::clear();
    if (!session || !negative) return invalid("a required pointer is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        auto t = parse_tier(tier);
        if (!t) fail_invalid("unknown tier");
        DeviceGuard dg(s.engine->device);
        TierState& ts = s.tier_source(*t);
        RenderCtx ctx{s.pool, s.stream};
        ctx.ae_ev = s.session_ev();
        ctx.pitch_um = s.tier_pitch_um(ts);
        const Size2 ns = prepared_size(s.params, ts.source.w, ts.source.h);
        const size_t cbytes = size_t(ns.w) * ns.h * 9 * sizeof(float);
        DevBuffer dc;
        if (counts) {
            dc = s.pool.acquire(cbytes);
            cuda_check(cudaMemsetAsync(dc.ptr(), 0, cbytes, s.stream), "memset");
        }
        Plane neg = develop(ctx, s.pipe, ts.source, seed, s.hal, counts ? dc.as<float>() : nullptr);
        cuda_check(cudaMemcpyAsync(negative, neg.data(), neg.bytes(), cudaMemcpyDeviceToHost, s.stream), "copy");
        if (counts) cuda_check(cudaMemcpyAsync(counts, dc.ptr(), cbytes, cudaMemcpyDeviceToHost, s.stream), "copy");
        cuda_check(cudaStreamSynchronize(s.stream), "develop");
        return SPK_OK;
    });
}

SPK_API spk_status spkx_session_develop_draws(spk_session* session, const char* tier, uint32_t seed, float* counts,
                                              float* lambdas) {
    last_error::clear();
    if (!session || !counts || !lambdas) return invalid("a required pointer is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        auto t = parse_tier(tier);
        if (!t) fail_invalid("unknown tier");
        DeviceGuard dg(s.engine->device);
        TierState& ts = s.tier_source(*t);
        RenderCtx ctx{s.pool, s.stream};
        ctx.ae_ev = s.session_ev();
        ctx.pitch_um = s.tier_pitch_um(ts);
        const Size2 ns = prepared_size(s.params, ts.source.w, ts.source.h);
        const size_t bytes = size_t(ns.w) * ns.h * 9 * sizeof(float);
        DevBuffer dc = s.pool.acquire(bytes), dl = s.pool.acquire(bytes);
        cuda_check(cudaMemsetAsync(dc.ptr(), 0, bytes, s.stream), "memset");
        cuda_check(cudaMemsetAsync(dl.ptr(), 0, bytes, s.stream), "memset");
        Plane neg = develop(ctx, s.pipe, ts.source, seed, s.hal, dc.as<float>(), dl.as<float>());
        cuda_check(cudaMemcpyAsync(counts, dc.ptr(), bytes, cudaMemcpyDeviceToHost, s.stream), "copy");
        cuda_check(cudaMemcpyAsync(lambdas, dl.ptr(), bytes, cudaMemcpyDeviceToHost, s.stream), "copy");
        cuda_check(cudaStreamSynchronize(s.stream), "develop");
        return SPK_OK;
    });
}

SPK_API spk_status spk_render_vjp(spk_session* session, const char* tier, uint32_t film_seed, const float* grad_output,
                                  float* grad_input, double* grad_params, uint32_t n_params, float* output) {
    last_error::clear();
    if (!session) return invalid("session is NULL");
    if (grad_output && !grad_input) return invalid("grad_input is NULL while grad_output is given");
    if (!grad_output && !output) return invalid("neither grad_output nor output is given");
    if (n_params > 0 && !grad_params) return invalid("grad_params is NULL with n_params > 0");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        auto t = parse_tier(tier);
        if (!t) fail_invalid("unknown tier");
        DeviceGuard dg(s.engine->device);
        TierState& ts = s.tier_source(*t);
        if (ts.source.w != s.source.w || ts.source.h != s.source.h)
            fail_unsupported("the render's adjoint runs on a tier whose image is the frame itself (no downscale)");
        RenderCtx ctx{s.pool, s.stream};
        ctx.pitch_um = s.tier_pitch_um(ts);
        const size_t bytes = s.source.pixels() * 3 * sizeof(float);
        DevBuffer dy, dgy, dgx;
        if (output) dy = s.pool.acquire(bytes);
        if (grad_output) {
            dgy = s.pool.acquire(bytes);
            dgx = s.pool.acquire(bytes);
            cuda_check(cudaMemcpyAsync(dgy.ptr(), grad_output, bytes, cudaMemcpyHostToDevice, s.stream), "copy");
        }
        render_vjp(ctx, s.pipe, s.live, s.source, film_seed, s.hal, output ? dy.as<float>() : nullptr,
                   grad_output ? dgy.as<float>() : nullptr, grad_output ? dgx.as<float>() : nullptr,
                   grad_output ? grad_params : nullptr, grad_output ? n_params : 0u);
        if (output) cuda_check(cudaMemcpyAsync(output, dy.ptr(), bytes, cudaMemcpyDeviceToHost, s.stream), "copy");
        if (grad_output)
            cuda_check(cudaMemcpyAsync(grad_input, dgx.ptr(), bytes, cudaMemcpyDeviceToHost, s.stream), "copy");
        cuda_check(cudaStreamSynchronize(s.stream), "render adjoint");
        cuda_check(cudaGetLastError(), "render adjoint");
        return SPK_OK;
    });
}

SPK_API spk_status spkx_session_setup_json(spk_session* session, double pitch_um, char** out_json) {
    last_error::clear();
    if (!session) return invalid("session is NULL");
    return guarded([&] {
        Session& s = *S(session);
        std::lock_guard<std::mutex> lock(s.m);
        put_json(out_json, setup_json(*s.pipe.film, *s.pipe.print, s.live, pitch_um));
        return SPK_OK;
    });
}

SPK_API spk_status spkx_setup_json(const char* resources_dir, const char* delta, double pitch_um, char** out_json) {
    last_error::clear();
    if (!resources_dir) return invalid("resources_dir is NULL");
    return guarded([&] {
        auto res = Resources::load(resources_dir);
        const Delta d = validate_delta(delta ? delta : "", DeltaContext::Open);
        std::shared_ptr<const Profile> film, print;
        const ParamSet p = open_params(*res, d, film, print);
        Cam16Cache cache;
        auto fs = build_film_setup(p, film, *res);
        auto ps = build_print_setup(p, *fs, print, *res, cache, !d.product_defaults.value_or(false));
        put_json(out_json, setup_json(*fs, *ps, LiveParams::from(p), pitch_um));
        return SPK_OK;
    });
}

}  // extern "C"

namespace {
template <class F>
spk_status with_scratch_stream(F&& f) {
    return guarded([&] {
        cudaStream_t s = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        try {
            f(s);
            cuda_check(cudaStreamSynchronize(s), "test kernel");
            cuda_check(cudaGetLastError(), "test kernel");
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
        return SPK_OK;
    });
}

struct DevArray {
    void* p = nullptr;
    explicit DevArray(size_t bytes) { cuda_check(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc"); }
    ~DevArray() { cudaFree(p); }
};
}  // namespace

extern "C" {

SPK_API spk_status spkx_sampler_poisson(const float* lam, float* counts, uint32_t n, uint32_t stream, uint32_t seed) {
    last_error::clear();
    if ((!lam || !counts) && n) return invalid("a required pointer is NULL");
    return with_scratch_stream([&](cudaStream_t s) {
        DevArray dl(n * 4ull), dc(n * 4ull);
        cuda_check(cudaMemcpyAsync(dl.p, lam, n * 4ull, cudaMemcpyHostToDevice, s), "copy");
        dev::sampler_poisson(static_cast<float*>(dl.p), static_cast<float*>(dc.p), n, stream, seed, s);
        cuda_check(cudaMemcpyAsync(counts, dc.p, n * 4ull, cudaMemcpyDeviceToHost, s), "copy");
        cuda_check(cudaStreamSynchronize(s), "sampler");
    });
}

SPK_API spk_status spkx_sampler_lognormal(float* out, uint32_t n, float mean, float stddev, uint32_t stream,
                                          uint32_t seed) {
    last_error::clear();
    if (!out && n) return invalid("out is NULL");
    return with_scratch_stream([&](cudaStream_t s) {
        DevArray d(n * 4ull);
        dev::sampler_lognormal(static_cast<float*>(d.p), n, mean, stddev, stream, seed, s);
        cuda_check(cudaMemcpyAsync(out, d.p, n * 4ull, cudaMemcpyDeviceToHost, s), "copy");
        cuda_check(cudaStreamSynchronize(s), "sampler");
    });
}

SPK_API spk_status spkx_philox(const uint32_t* counters, const uint32_t* keys, uint32_t* out, uint32_t n) {
    last_error::clear();
    if ((!counters || !keys || !out) && n) return invalid("a required pointer is NULL");
    return with_scratch_stream([&](cudaStream_t s) {
        DevArray dc(n * 16ull), dk(n * 8ull), dout(n * 16ull);
        cuda_check(cudaMemcpyAsync(dc.p, counters, n * 16ull, cudaMemcpyHostToDevice, s), "copy");
        cuda_check(cudaMemcpyAsync(dk.p, keys, n * 8ull, cudaMemcpyHostToDevice, s), "copy");
        dev::philox_blocks(static_cast<uint32_t*>(dc.p), static_cast<uint32_t*>(dk.p), static_cast<uint32_t*>(dout.p),
                           n, s);
        cuda_check(cudaMemcpyAsync(out, dout.p, n * 16ull, cudaMemcpyDeviceToHost, s), "copy");
        cuda_check(cudaStreamSynchronize(s), "philox");
    });
}

SPK_API spk_status spkx_test_set_tc_wait_limit(int64_t cycles) {
    last_error::clear();
    if (cycles < 0) return invalid("a wait limit is a count of SM clocks, 0 or more");
    dev::set_tc_wait_limit(cycles);
    return SPK_OK;
}

SPK_API spk_status spkx_test_set_iir_wait_limit(int64_t cycles) {
    last_error::clear();
    if (cycles < 0) return invalid("a wait limit is a count of SM clocks, 0 or more");
    dev::set_iir_wait_limit(cycles);
    return SPK_OK;
}

SPK_API spk_status spkx_test_take_iir_waits_given_up(uint32_t* count) {
    last_error::clear();
    if (!count) return invalid("count is NULL");
    return with_scratch_stream([&](cudaStream_t s) { *count = dev::take_iir_waits_given_up(s); });
}

SPK_API spk_status spkx_gaussian(const float* in, float* out, uint32_t w, uint32_t h, const double* sigma3) {
    last_error::clear();
    if (!in || !out || !sigma3) return invalid("a required pointer is NULL");
    if (w == 0 || h == 0) return invalid("empty plane");
    return with_scratch_stream([&](cudaStream_t s) {
        Pool pool(s);
        RenderCtx ctx{pool, s};
        Plane a = make_plane(pool, w, h), b = make_plane(pool, w, h);
        cuda_check(cudaMemcpyAsync(a.data(), in, a.bytes(), cudaMemcpyHostToDevice, s), "copy");
        gaussian(ctx, a, b, Vec3{sigma3[0], sigma3[1], sigma3[2]});
        cuda_check(cudaMemcpyAsync(out, b.data(), b.bytes(), cudaMemcpyDeviceToHost, s), "copy");
        cuda_check(cudaStreamSynchronize(s), "gaussian");
    });
}

}  // extern "C"
