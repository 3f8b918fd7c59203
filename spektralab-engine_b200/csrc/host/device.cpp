#include "device.hpp"

#include <vector>

#include "status.hpp"

namespace spkb {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail_gpu(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

struct PoolState {
    mutable std::mutex m;
    std::multimap<size_t, void*> free;
    size_t live = 0, idle = 0;
    ~PoolState() {
        for (auto& [sz, p] : free) cudaFree(p);
    }
};

struct DevBuffer::Impl {
    void* p = nullptr;
    size_t size = 0;
    std::shared_ptr<PoolState> pool;  // null: persistent
    ~Impl() {
        if (!p) return;
        if (pool) {
            std::lock_guard<std::mutex> g(pool->m);
            pool->free.emplace(size, p);
            pool->live -= size;
            pool->idle += size;
        } else {
            cudaFree(p);
        }
    }
};

void* DevBuffer::ptr() const { return p_ ? p_->p : nullptr; }
size_t DevBuffer::size() const { return p_ ? p_->size : 0; }

Pool::Pool() : s_(std::make_shared<PoolState>()) {}

DevBuffer Pool::acquire(size_t bytes) {
    bytes = std::max<size_t>((bytes + 255) / 256 * 256, 256);
    void* p = nullptr;
    size_t size = 0;
    {
        std::lock_guard<std::mutex> g(s_->m);
        auto it = s_->free.lower_bound(bytes);
        if (it != s_->free.end() && it->first <= 2 * bytes) {
            size = it->first;
            p = it->second;
            s_->free.erase(it);
            s_->idle -= size;
        }
    }
    if (!p) {
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            trim();
            cuda_check(cudaMalloc(&p, bytes), "cudaMalloc (scratch)");
        }
        size = bytes;
    }
    {
        std::lock_guard<std::mutex> g(s_->m);
        s_->live += size;
    }
    auto impl = std::make_shared<DevBuffer::Impl>();
    impl->p = p;
    impl->size = size;
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
        trim();
        cuda_check(cudaMalloc(&p, bytes), "cudaMalloc (persistent)");
    }
    auto impl = std::make_shared<DevBuffer::Impl>();
    impl->p = p;
    impl->size = bytes;
    DevBuffer b;
    b.p_ = std::move(impl);
    return b;
}

size_t Pool::trim() {
    std::lock_guard<std::mutex> g(s_->m);
    size_t freed = 0;
    for (auto& [sz, p] : s_->free) {
        cudaFree(p);
        freed += sz;
    }
    s_->free.clear();
    s_->idle = 0;
    return freed;
}

size_t Pool::live_bytes() const {
    std::lock_guard<std::mutex> g(s_->m);
    return s_->live;
}
size_t Pool::free_bytes() const {
    std::lock_guard<std::mutex> g(s_->m);
    return s_->idle;
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
