#include "device.hpp"

#include <atomic>
#include <cstdint>
#include <vector>

#include "status.hpp"

namespace spkb {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail_gpu(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

struct PoolState {
    std::mutex m;
    cudaStream_t stream = nullptr;
    size_t live = 0;
};

namespace {
// process-wide allocation counters behind the memory report
std::atomic<uint64_t> g_scratch_allocations{0}, g_scratch_live{0}, g_persistent_allocations{0};
std::atomic<uint64_t> g_persistent_live{0}, g_persistent_bytes{0};
}  // namespace

struct DevBuffer::Impl {
    void* p = nullptr;
    size_t size = 0;
    std::shared_ptr<PoolState> pool;  // null: persistent (cudaMalloc)
    ~Impl() {
        if (!p) return;
        if (pool) {
            std::lock_guard<std::mutex> g(pool->m);
            cudaFreeAsync(p, pool->stream);
            pool->live -= size;
            g_scratch_live.fetch_sub(1);
        } else {
            g_persistent_live.fetch_sub(1);
            g_persistent_bytes.fetch_sub(size);
            cudaFree(p);
        }
    }
};

void* DevBuffer::ptr() const { return p_ ? p_->p : nullptr; }
size_t DevBuffer::size() const { return p_ ? p_->size : 0; }

Pool::Pool(cudaStream_t stream) : s_(std::make_shared<PoolState>()) { s_->stream = stream; }

void Pool::set_stream(cudaStream_t s) {
    std::lock_guard<std::mutex> g(s_->m);
    s_->stream = s;
}

cudaStream_t Pool::stream() const { return s_->stream; }

DevBuffer Pool::acquire(size_t bytes) {
    bytes = std::max<size_t>((bytes + 255) / 256 * 256, 256);
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, s_->stream);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        int dev = 0;
        cudaGetDevice(&dev);
        cudaStreamSynchronize(s_->stream);
        device_pool_trim(dev);
        cuda_check(cudaMallocAsync(&p, bytes, s_->stream), "cudaMallocAsync (scratch)");
    }
    {
        std::lock_guard<std::mutex> g(s_->m);
        s_->live += bytes;
    }
    g_scratch_allocations.fetch_add(1);
    g_scratch_live.fetch_add(1);
    auto impl = std::make_shared<DevBuffer::Impl>();
    impl->p = p;
    impl->size = bytes;
    impl->pool = s_;
    DevBuffer b;
    b.p_ = std::move(impl);
    return b;
}

DevBuffer Pool::persistent(size_t bytes) {
    void* p = nullptr;
    bytes = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        int dev = 0;
        cudaGetDevice(&dev);
        device_pool_trim(dev);
        cuda_check(cudaMalloc(&p, bytes), "cudaMalloc (persistent)");
    }
    g_persistent_allocations.fetch_add(1);
    g_persistent_live.fetch_add(1);
    g_persistent_bytes.fetch_add(bytes);
    auto impl = std::make_shared<DevBuffer::Impl>();
    impl->p = p;
    impl->size = bytes;
    DevBuffer b;
    b.p_ = std::move(impl);
    return b;
}

size_t Pool::live_bytes() const {
    std::lock_guard<std::mutex> g(s_->m);
    return s_->live;
}

void configure_device_pool(int device) {
    cudaMemPool_t mp = nullptr;
    cuda_check(cudaDeviceGetDefaultMemPool(&mp, device), "cudaDeviceGetDefaultMemPool");
    uint64_t threshold = UINT64_MAX;
    cuda_check(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
}

size_t device_pool_reserved(int device) {
    cudaMemPool_t mp = nullptr;
    if (cudaDeviceGetDefaultMemPool(&mp, device) != cudaSuccess) return 0;
    uint64_t v = 0;
    cudaMemPoolGetAttribute(mp, cudaMemPoolAttrReservedMemCurrent, &v);
    return size_t(v);
}

DeviceMemory device_memory(int device) {
    DeviceMemory m;
    cudaMemPool_t mp = nullptr;
    if (cudaDeviceGetDefaultMemPool(&mp, device) == cudaSuccess) {
        uint64_t v = 0;
        if (cudaMemPoolGetAttribute(mp, cudaMemPoolAttrReservedMemCurrent, &v) == cudaSuccess) m.reserved = v;
        if (cudaMemPoolGetAttribute(mp, cudaMemPoolAttrUsedMemCurrent, &v) == cudaSuccess) m.used = v;
        if (cudaMemPoolGetAttribute(mp, cudaMemPoolAttrUsedMemHigh, &v) == cudaSuccess) m.used_high = v;
    }
    m.scratch_allocations = g_scratch_allocations.load();
    m.scratch_live = g_scratch_live.load();
    m.persistent_allocations = g_persistent_allocations.load();
    m.persistent_live = g_persistent_live.load();
    m.persistent_bytes = g_persistent_bytes.load();
    return m;
}

void device_pool_begin_frame(int device) {
    cudaMemPool_t mp = nullptr;
    if (cudaDeviceGetDefaultMemPool(&mp, device) != cudaSuccess) return;
    uint64_t zero = 0;
    (void)cudaMemPoolSetAttribute(mp, cudaMemPoolAttrUsedMemHigh, &zero);
}

size_t device_pool_trim(int device) {
    cudaMemPool_t mp = nullptr;
    if (cudaDeviceGetDefaultMemPool(&mp, device) != cudaSuccess) return 0;
    const size_t before = device_pool_reserved(device);
    cudaMemPoolTrimTo(mp, 0);
    const size_t after = device_pool_reserved(device);
    return before > after ? before - after : 0;
}

// ---- result images -------------------------------------------------------------------------------

namespace {
struct OutputCache {
    std::mutex m;
    std::multimap<std::pair<int, size_t>, OutputImage*> idle;  // (device, bytes)
};
OutputCache& output_cache() {
    static OutputCache* c = new OutputCache();  // process lifetime: results outlive every engine
    return *c;
}
struct PinnedCache {
    std::mutex m;
    std::multimap<size_t, void*> idle;
};
PinnedCache& pinned_cache() {
    static PinnedCache* c = new PinnedCache();
    return *c;
}
}  // namespace

OutputImage* output_acquire(int device, uint32_t w, uint32_t h) {
    const uint32_t stride = (w + kOutputRowAlignPx - 1) / kOutputRowAlignPx * kOutputRowAlignPx;
    const size_t bytes = size_t(stride) * 8 * h;
    OutputCache& c = output_cache();
    {
        std::lock_guard<std::mutex> g(c.m);
        auto it = c.idle.find({device, bytes});
        if (it != c.idle.end()) {
            OutputImage* img = it->second;
            c.idle.erase(it);
            img->width = w;
            img->height = h;
            img->stride_px = stride;
            return img;
        }
    }
    auto* img = new OutputImage();
    img->bytes = bytes;
    img->width = w;
    img->height = h;
    img->stride_px = stride;
    img->device = device;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&img->dev), bytes);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&img->host), bytes);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        if (img->dev) cudaFree(img->dev);
        delete img;
        output_trim();
        fail_gpu(std::string("cannot allocate the output image: ") + cudaGetErrorName(e));
    }
    return img;
}

void output_release(OutputImage* img) {
    if (!img) return;
    OutputCache& c = output_cache();
    std::lock_guard<std::mutex> g(c.m);
    c.idle.emplace(std::make_pair(img->device, img->bytes), img);
}

size_t output_trim() {
    OutputCache& c = output_cache();
    std::lock_guard<std::mutex> g(c.m);
    size_t freed = 0;
    for (auto& [k, img] : c.idle) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(img->device);
        cudaFree(img->dev);
        cudaFreeHost(img->host);
        cudaSetDevice(cur);
        freed += img->bytes;
        delete img;
    }
    c.idle.clear();
    return freed;
}

PinnedBuffer pinned_acquire(size_t bytes) {
    PinnedCache& c = pinned_cache();
    {
        std::lock_guard<std::mutex> g(c.m);
        auto it = c.idle.lower_bound(bytes);
        if (it != c.idle.end() && it->first <= 2 * bytes) {
            PinnedBuffer b{it->second, it->first};
            c.idle.erase(it);
            return b;
        }
    }
    PinnedBuffer b;
    b.bytes = bytes;
    cuda_check(cudaMallocHost(&b.p, bytes), "cudaMallocHost (input staging)");
    return b;
}

void pinned_release(PinnedBuffer b) {
    if (!b.p) return;
    PinnedCache& c = pinned_cache();
    std::lock_guard<std::mutex> g(c.m);
    c.idle.emplace(b.bytes, b.p);
}

}  // namespace spkb
