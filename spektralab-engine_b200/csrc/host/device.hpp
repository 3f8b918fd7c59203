// Device memory and streams of the B200 engine.
//
//   Pool        per session: scratch buffers from CUDA's stream-ordered allocator (cudaMallocAsync on the
//               session's stream, from the device's memory pool, which keeps freed memory cached), so a
//               plane freed by one stage is reused by the next on the same stream with no
//               synchronisation and a new session allocates from the cache.
//   persistent  tables that can outlive a session (cached pipelines): plain cudaMalloc / cudaFree.
//   DevBuffer   a handle; dropping the last copy frees the memory (stream-ordered for scratch).
//   Plane       interleaved binary32 RGB in device memory.
//   OutputImage a rendered RGBA16 image: a device copy and a pinned host copy, drawn from a process-wide
//               cache so that a result outlives its session and engine and pinning is paid once.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>

namespace spkb {

void cuda_check(cudaError_t e, const char* what);  // throws SPK_ERR_GPU

struct PoolState;

class DevBuffer {
public:
    DevBuffer() = default;
    explicit operator bool() const { return p_ != nullptr; }
    void* ptr() const;
    size_t size() const;
    template <class T>
    T* as() const { return static_cast<T*>(ptr()); }

private:
    friend class Pool;
    struct Impl;
    std::shared_ptr<Impl> p_;
};

class Pool {
public:
    explicit Pool(cudaStream_t stream = nullptr);
    void set_stream(cudaStream_t s);
    cudaStream_t stream() const;
    DevBuffer acquire(size_t bytes);          // stream-ordered device memory, contents undefined
    DevBuffer persistent(size_t bytes);       // cudaMalloc'd: may outlive the stream
    size_t live_bytes() const;                // bytes of this pool's live scratch buffers

private:
    std::shared_ptr<PoolState> s_;
};

// The device memory pool behind every Pool: keep all freed memory cached (release threshold max).
void configure_device_pool(int device);
size_t device_pool_trim(int device);          // returns the cached bytes released to the driver
size_t device_pool_reserved(int device);

// The figures behind the memory report: the device pool's reserved and used bytes and its used high-water
// mark (cudaMemPoolAttr*), and this process's scratch and persistent allocation counters.
struct DeviceMemory {
    uint64_t reserved = 0, used = 0, used_high = 0;
    uint64_t scratch_allocations = 0, scratch_live = 0;
    uint64_t persistent_allocations = 0, persistent_live = 0, persistent_bytes = 0;
};
DeviceMemory device_memory(int device);
// A render begins: the pool's used high-water mark starts again from the bytes in use.
void device_pool_begin_frame(int device);

struct Plane {
    DevBuffer buf;
    uint32_t w = 0, h = 0;
    explicit operator bool() const { return static_cast<bool>(buf); }
    float* data() const { return buf.as<float>(); }
    size_t pixels() const { return size_t(w) * h; }
    size_t bytes() const { return pixels() * 3 * sizeof(float); }
};

inline Plane make_plane(Pool& pool, uint32_t w, uint32_t h) {
    Plane p;
    p.w = w;
    p.h = h;
    p.buf = pool.acquire(size_t(w) * h * 3 * sizeof(float));
    return p;
}

// The result image behind spk_result.texture.
struct OutputImage {
    uint16_t* dev = nullptr;   // RGBA16, row pitch stride_px pixels
    uint16_t* host = nullptr;  // pinned
    size_t bytes = 0;
    uint32_t width = 0, height = 0, stride_px = 0;
    int device = 0;
};
constexpr uint32_t kOutputRowAlignPx = 32;  // 256-byte rows
OutputImage* output_acquire(int device, uint32_t w, uint32_t h);
void output_release(OutputImage* img);
size_t output_trim();

// Pinned host staging for host inputs (spk_open's frame upload), process-wide and reused.
struct PinnedBuffer {
    void* p = nullptr;
    size_t bytes = 0;
};
PinnedBuffer pinned_acquire(size_t bytes);
void pinned_release(PinnedBuffer b);

}  // namespace spkb
