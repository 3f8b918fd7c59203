// spkx_gaussian_noalloc: the Gaussian blur of a device plane with no device allocation at all.
//
// Some hosts cannot let a plug-in allocate device memory while they call it: a video or photo editor
// that hands the plug-in its frame buffers inside a per-frame render callback, with the card's memory
// already budgeted up front by the host's own allocator, or a real-time pipeline where cudaMalloc's
// latency and implicit synchronisation are not allowed. They pass their own input and output buffers;
// the one intermediate plane this blur needs lives in a fixed array compiled into the library.
//
// The scratch is a file-scope __device__ array of two planes of kMaxFloats floats each (16 MiB in all),
// so a frame of at most kMaxFloats / 3 pixels (699,050, e.g. 1024 x 682). Every GPU that loads the
// library holds the array until the process exits. Host code cannot use the array's name as a device
// address (it is a host-side stand-in), so the first call in each CUDA context, with that context current,
// looks the address up with cudaGetSymbolAddress and keeps it for later calls in the same context; make
// that first call before any stream capture. The address belongs to the context it was looked up in: a
// host that makes its own driver contexts current, or resets the device, gets a fresh lookup for each new
// context (the cache is keyed by the driver's unique context id). Every call in a context shares the
// array, which keeps whatever the last call left in it: calls whose work overlaps on the GPU (different
// streams, or a later call before an earlier one's work has finished on another stream) race on it.
// Nothing has to start at zero: each pass writes every scratch element it later reads.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../host/blur_plan.h"
#include "../host/status.hpp"
#include "launch.hpp"
#include "spektralab_b200.h"

namespace spkb::dev {
namespace {

constexpr size_t kMaxFloats = size_t(1) << 21;  // one plane: 2,097,152 floats (8 MiB)
__device__ __align__(256) float g_scratch[2 * kMaxFloats];

std::mutex g_mutex;
std::vector<std::pair<unsigned long long, float*>> g_address;  // (driver context id, address of g_scratch)

// The device address of g_scratch in the current context, looked up once per context. The caller holds
// g_mutex.
float* scratch_address(cudaError_t* err) {
    unsigned long long id = current_context_id();
    for (const auto& [ctx, p] : g_address)
        if (id != 0 && ctx == id) return p;
    void* p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_scratch);  // makes the device's primary context current if none is
    if (*err != cudaSuccess) return nullptr;
    if (id == 0) id = current_context_id();
    if (id == 0) {
        *err = cudaErrorDeviceUninitialized;
        return nullptr;
    }
    if (g_address.size() >= 256) g_address.clear();  // a host that cycles through contexts: forget the old
    g_address.emplace_back(id, static_cast<float*>(p));
    return static_cast<float*>(p);
}

}  // namespace
}  // namespace spkb::dev

using namespace spkb;

extern "C" SPK_API spk_status spkx_gaussian_noalloc(const float* in, float* out, uint32_t w, uint32_t h,
                                                    const double* sigma3, void* stream) {
    last_error::clear();
    if (!in || !out || !sigma3) {
        last_error::set("a required pointer is NULL");
        return SPK_ERR_INVALID_ARG;
    }
    if (w == 0 || h == 0) {
        last_error::set("empty plane");
        return SPK_ERR_INVALID_ARG;
    }
    const size_t floats = size_t(w) * h * 3;
    if (floats > dev::kMaxFloats) {
        last_error::set("spkx_gaussian_noalloc: a " + std::to_string(w) + " x " + std::to_string(h) +
                        " plane needs " + std::to_string(floats) + " scratch floats; the fixed scratch holds " +
                        std::to_string(dev::kMaxFloats) + " (at most " + std::to_string(dev::kMaxFloats / 3) +
                        " pixels)");
        return SPK_ERR_INVALID_ARG;
    }
    cudaError_t e = cudaSuccess;
    float* s0 = nullptr;
    {
        std::lock_guard<std::mutex> lock(dev::g_mutex);
        s0 = dev::scratch_address(&e);
    }
    if (!s0) {
        last_error::set(std::string("spkx_gaussian_noalloc: no scratch address in the current CUDA context: ") +
                        cudaGetErrorString(e));
        return SPK_ERR_GPU;
    }
    float* s1 = s0 + dev::kMaxFloats;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    bool iir[3];
    int n_iir = 0;
    for (int c = 0; c < 3; ++c) {
        iir[c] = blur_branch_code(sigma3[c]) == BLUR_IIR;
        n_iir += iir[c];
    }
    const FirTaps taps = blur_fir_taps(sigma3, iir);
    const float one[3] = {1.0f, 1.0f, 1.0f};
    if (n_iir == 0) {
        if (taps.r == 0) {
            if (in != out) dev::copy(in, out, size_t(w) * h, st);
        } else {
            dev::fir_v(in, s0, w, h, taps, st);
            dev::fir_h(s0, out, out, w, h, taps, ACC_NONE, one, st);
        }
    } else {
        const float* src = in;
        if (n_iir < 3 && taps.r > 0) {  // FIR channels first, the recursive ones pass through as a delta
            dev::fir_v(in, s0, w, h, taps, st);
            dev::fir_h(s0, s1, s1, w, h, taps, ACC_NONE, one, st);
            src = s1;
        }
        // the block-parallel kernels where the lines fit in shared memory (the other channels pass
        // through), else one thread per line
        if (!blur_iir_block(src, out, s0, w, h, sigma3, iir, st)) {
            const IirCoefs coefs = blur_iir_coefs(sigma3, iir);
            dev::iir_h(src, s0, w, h, coefs, st);
            dev::iir_v(s0, out, out, w, h, coefs, ACC_NONE, one, st);
        }
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        last_error::set(std::string("spkx_gaussian_noalloc: ") + cudaGetErrorString(e));
        return SPK_ERR_GPU;
    }
    return SPK_OK;
}
