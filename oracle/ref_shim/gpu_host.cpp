// Test infrastructure (oracle): a host implementation of the reference engine's GPU layer
// (src/gpu/gpu.hpp of the reference), so that its stage code in src/film, src/print, src/fx and
// src/session runs unmodified on CPU cores. It replaces the Objective-C++ Metal bridge (src/gpu/gpu.mm).
//
//   Buffer   64-byte aligned host memory; pooled buffers return to their Pool when the last handle drops
//   Pool     reuse rule of the reference (src/gpu/gpu.mm:125-161): the smallest free buffer in [b, 2b]
//   Batch    each dispatch runs at once over its grid (OpenMP), in encode order; commit_and_wait is a no-op
//   Kernel   looked up by name in the registry of kernels/*.metal compiled as C++ (kernel_registry.hpp)
//   output   RGBA16 rows padded to 256 bytes (32 pixels), the "texture" is a host allocation
//   probe    the reference's spk_probe_fma under this build's flags (no contraction, no fast math)
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gpu/gpu.hpp"
#include "kernel_registry.hpp"
#include "util/error.hpp"

namespace spkref {

namespace {
std::map<std::string, KernelInfo>& registry() {
    static std::map<std::string, KernelInfo> r;
    return r;
}
}  // namespace

void register_kernel(const char* name, KernelThunk run, int dims) { registry()[name] = KernelInfo{run, dims}; }

const KernelInfo* find_kernel(const std::string& name) {
    auto it = registry().find(name);
    return it == registry().end() ? nullptr : &it->second;
}

}  // namespace spkref

namespace spk::gpu {

namespace {
constexpr size_t kAlign = 64;
constexpr size_t kOutputRowAlignBytes = 256;

void* host_alloc(size_t bytes) {
    void* p = std::aligned_alloc(kAlign, std::max<size_t>((bytes + kAlign - 1) / kAlign * kAlign, kAlign));
    if (!p) throw std::bad_alloc();
    return p;
}
}  // namespace

struct LedgerState {
    std::mutex m;
    PersistentStats st;
};

struct PoolState {
    std::mutex m;
    std::multimap<size_t, void*> free;  // size -> memory
    PoolStats st;
};

struct BufferImpl {
    void* mem = nullptr;
    size_t size = 0;
    bool owned = true;
    std::shared_ptr<PoolState> pool;      // set for pooled buffers
    std::shared_ptr<LedgerState> ledger;  // set for persistent buffers
    MemTag tag = MemTag::Other;
    ~BufferImpl() {
        if (!owned || !mem) return;
        if (pool) {
            std::lock_guard<std::mutex> g(pool->m);
            pool->free.emplace(size, mem);
            pool->st.live_bytes -= size;
            pool->st.free_bytes += size;
            --pool->st.live_buffers;
            ++pool->st.free_buffers;
            return;
        }
        if (ledger) {
            std::lock_guard<std::mutex> g(ledger->m);
            ledger->st.bytes -= size;
            --ledger->st.buffers;
            ledger->st.by_tag[size_t(tag)] -= size;
        }
        std::free(mem);
    }
};

struct ContextImpl {
    std::string name = "host CPU (reference oracle)";
};

struct ArgAccess {
    static bool is_buffer(const Arg& a) { return a.kind_ == Arg::Kind::Buf; }
    static const Buffer& buffer(const Arg& a) { return a.buf_; }
    static size_t offset(const Arg& a) { return a.off_; }
    static const std::vector<uint8_t>& bytes(const Arg& a) { return a.bytes_; }
};

struct Batch::Impl {
    bool used = false;
};

// ---- Buffer --------------------------------------------------------------------------------------
void* Buffer::contents() const { return p_ ? p_->mem : nullptr; }
size_t Buffer::size() const { return p_ ? p_->size : 0; }
void* Buffer::mtl() const { return p_ ? p_->mem : nullptr; }
bool Buffer::pooled() const { return p_ && p_->pool; }

// ---- Pool ----------------------------------------------------------------------------------------
Buffer Pool::acquire(size_t bytes) {
    if (!s_) s_ = std::make_shared<PoolState>();
    bytes = std::max<size_t>(bytes, 4);
    void* mem = nullptr;
    size_t size = 0;
    {
        std::lock_guard<std::mutex> g(s_->m);
        auto it = s_->free.lower_bound(bytes);
        if (it != s_->free.end() && it->first <= 2 * bytes) {
            size = it->first;
            mem = it->second;
            s_->free.erase(it);
            s_->st.free_bytes -= size;
            --s_->st.free_buffers;
            ++s_->st.reuses;
        }
    }
    if (!mem) {
        mem = host_alloc(bytes);
        size = bytes;
        std::lock_guard<std::mutex> g(s_->m);
        s_->st.total_bytes += size;
        ++s_->st.buffers;
        ++s_->st.allocations;
    }
    {
        std::lock_guard<std::mutex> g(s_->m);
        s_->st.live_bytes += size;
        ++s_->st.live_buffers;
        s_->st.frame_high_water_bytes = std::max(s_->st.frame_high_water_bytes, s_->st.live_bytes);
    }
    auto impl = std::make_shared<BufferImpl>();
    impl->mem = mem;
    impl->size = size;
    impl->pool = s_;
    Buffer b;
    b.p_ = std::move(impl);
    return b;
}

Plane Pool::plane(uint32_t w, uint32_t h) {
    Plane p;
    p.w = w;
    p.h = h;
    p.buf = acquire(size_t(w) * h * Plane::kChannels * sizeof(float));
    return p;
}

size_t Pool::trim(size_t keep_bytes) {
    if (!s_) return 0;
    std::lock_guard<std::mutex> g(s_->m);
    size_t freed = 0;
    while (s_->st.free_bytes > keep_bytes && !s_->free.empty()) {
        auto it = std::prev(s_->free.end());
        std::free(it->second);
        freed += it->first;
        s_->st.free_bytes -= it->first;
        s_->st.total_bytes -= it->first;
        --s_->st.free_buffers;
        --s_->st.buffers;
        s_->free.erase(it);
    }
    return freed;
}

void Pool::begin_frame() {
    if (!s_) return;
    std::lock_guard<std::mutex> g(s_->m);
    s_->st.frame_high_water_bytes = s_->st.live_bytes;
}

PoolStats Pool::stats() const {
    if (!s_) return {};
    std::lock_guard<std::mutex> g(s_->m);
    return s_->st;
}

// ---- Batch ---------------------------------------------------------------------------------------
Batch::Batch(Batch&&) noexcept = default;
Batch& Batch::operator=(Batch&&) noexcept = default;
Batch::~Batch() = default;

namespace {
void run_kernel(const Kernel& k, uint32_t gx, uint32_t gy, const Arg* args, size_t n, int dims) {
    const spkref::KernelInfo* info = spkref::find_kernel(k.name());
    if (!info) fail_gpu("kernel '" + k.name() + "' is not in the host kernel registry");
    if (info->dims != dims) fail_gpu("kernel '" + k.name() + "' dispatched with the wrong grid rank");
    std::vector<void*> slots(n);
    for (size_t i = 0; i < n; ++i) {
        const Arg& a = args[i];
        if (ArgAccess::is_buffer(a)) {
            slots[i] = static_cast<uint8_t*>(ArgAccess::buffer(a).contents()) + ArgAccess::offset(a);
        } else {
            slots[i] = const_cast<uint8_t*>(ArgAccess::bytes(a).data());
        }
    }
    info->run(slots.data(), gx, gy);
}
}  // namespace

void Batch::dispatch_1d(const Kernel& k, uint32_t n, std::initializer_list<Arg> args) {
    p_->used = true;
    run_kernel(k, n, 1, args.begin(), args.size(), 1);
}
void Batch::dispatch_2d(const Kernel& k, uint32_t w, uint32_t h, std::initializer_list<Arg> args) {
    p_->used = true;
    run_kernel(k, w, h, args.begin(), args.size(), 2);
}
void Batch::dispatch_1d(const Kernel& k, uint32_t n, const std::vector<Arg>& args) {
    p_->used = true;
    run_kernel(k, n, 1, args.data(), args.size(), 1);
}
void Batch::dispatch_2d(const Kernel& k, uint32_t w, uint32_t h, const std::vector<Arg>& args) {
    p_->used = true;
    run_kernel(k, w, h, args.data(), args.size(), 2);
}
void Batch::commit_and_wait() {}
bool Batch::empty() const { return !p_ || !p_->used; }

// ---- Context -------------------------------------------------------------------------------------
std::shared_ptr<Context> Context::create(void*, const std::filesystem::path&) {
    std::shared_ptr<Context> c(new Context());
    c->p_ = std::make_unique<ContextImpl>();
    c->ledger_ = std::make_shared<LedgerState>();
    c->pool_.s_ = std::make_shared<PoolState>();
    return c;
}
Context::~Context() = default;
void* Context::device() const { return nullptr; }
std::string Context::device_name() const { return p_->name; }
uint32_t Context::max_texture_dimension_2d() const { return 16384; }
size_t Context::linear_texture_alignment_rgba16() const { return kOutputRowAlignBytes; }

Kernel Context::kernel(std::string_view name) {
    const spkref::KernelInfo* info = spkref::find_kernel(std::string(name));
    if (!info) fail_gpu("kernel '" + std::string(name) + "' is not in the host kernel registry");
    Kernel k;
    k.name_ = std::string(name);
    k.pso_ = reinterpret_cast<void*>(info->run);
    k.tew_ = 32;
    k.max_threads_ = 1024;
    return k;
}

Batch Context::batch() {
    Batch b;
    b.p_ = std::make_unique<Batch::Impl>();
    return b;
}

Buffer Context::persistent(size_t bytes, MemTag tag) {
    auto impl = std::make_shared<BufferImpl>();
    impl->mem = host_alloc(bytes);
    impl->size = bytes;
    impl->ledger = ledger_;
    impl->tag = tag;
    {
        std::lock_guard<std::mutex> g(ledger_->m);
        ledger_->st.bytes += bytes;
        ++ledger_->st.buffers;
        ledger_->st.by_tag[size_t(tag)] += bytes;
    }
    Buffer b;
    b.p_ = std::move(impl);
    return b;
}

Plane Context::persistent_plane(uint32_t w, uint32_t h, MemTag tag) {
    Plane p;
    p.w = w;
    p.h = h;
    p.buf = persistent(size_t(w) * h * Plane::kChannels * sizeof(float), tag);
    return p;
}

PersistentStats Context::persistent_stats() const {
    std::lock_guard<std::mutex> g(ledger_->m);
    return ledger_->st;
}

void Context::note_file_backed(size_t bytes) {
    std::lock_guard<std::mutex> g(ledger_->m);
    ledger_->st.bytes += bytes;
    ++ledger_->st.buffers;
    ledger_->st.file_backed_bytes += bytes;
    ++ledger_->st.file_backed_buffers;
    ledger_->st.by_tag[size_t(MemTag::Table)] += bytes;
}

// A "device buffer" for spk_open_device on this host build is any host allocation whose first
// 8 bytes are not inspected: the caller passes a pointer and the session checks the length it needs
// against buffer_length, which this build cannot know, so device inputs are refused.
Buffer Context::wrap(void*) { fail_gpu("device buffers are not supported by the host oracle build"); }
bool Context::same_device(void*) const { return false; }
size_t Context::buffer_length(void*) { return 0; }

namespace {
struct HostTexture {
    uint16_t* pixels = nullptr;
    ~HostTexture() { std::free(pixels); }
};
}  // namespace

OutputImage Context::make_output(uint32_t width, uint32_t height) {
    if (width == 0 || height == 0) fail_gpu("empty output image");
    const size_t a = kOutputRowAlignBytes / 8;
    const size_t stride = (size_t(width) + a - 1) / a * a;
    auto* t = new HostTexture();
    t->pixels = static_cast<uint16_t*>(host_alloc(stride * 8 * height));
    OutputImage out;
    out.texture = t;
    out.rgba16 = t->pixels;
    out.width = width;
    out.height = height;
    out.row_stride_px = uint32_t(stride);
    return out;
}

void Context::finish_output(const OutputImage&) {}

void Context::release_texture(void* texture) { delete static_cast<HostTexture*>(texture); }

ProbeResult Context::probe_math_mode() {
    constexpr uint32_t n = 64;
    ProbeResult r;
    Buffer a = pool_.acquire(n * sizeof(float));
    Buffer b = pool_.acquire(n * sizeof(float));
    Buffer o = pool_.acquire(n * sizeof(float));
    float* pa = a.as<float>();
    float* pb = b.as<float>();
    for (uint32_t i = 0; i < n; ++i) {
        pa[i] = static_cast<float>(0.1 + 0.37 * double(i));
        pb[i] = 0.5f * pa[i] + 1.0f;
    }
    std::memset(o.contents(), 0xFF, n * sizeof(float));
    Batch bt = batch();
    bt.dispatch_1d(kernel("spk_probe_fma"), n, {Arg::buffer(a), Arg::buffer(b), Arg::buffer(o), Arg::value(n)});
    bt.commit_and_wait();
    // This host build compiles every kernel with -ffp-contract=off and no fast math (oracle/Makefile), so
    // a*b - a*b is exactly 0 here; the Metal probe's FMA-contraction test has no host counterpart.
    const float* po = o.as<float>();
    uint32_t exact = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (po[i] == 0.0f) ++exact;
    }
    r.ok = exact == n;
    r.verdict = r.ok ? "safe (host build: -ffp-contract=off, no fast math)" : "unknown (host probe)";
    if (!r.ok) r.detail = "host probe: " + std::to_string(exact) + "/64 values are exactly a*b - a*b";
    return r;
}

}  // namespace spk::gpu
