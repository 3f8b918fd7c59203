// The block-parallel recursive Gaussian mixture (iir.cu): arguments and launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"
#include "launch.hpp"

namespace spkb::dev {

constexpr int kIirScanSteps = 7;  // carries of up to 2^7 segments per line

// One channel of one component: Young-van Vliet coefficients and the powers M^(2^p), p = 0..6, of M,
// the map of a segment's entry state (w[i-1], w[i-2], w[i-3]) through seg_len steps of the homogeneous
// recurrence (the parallel scan of the segment carries applies M^(2^p) at step p).
struct IirChannel {
    double B, B1, B2, B3;
    double Mp[kIirScanSteps][3][3];
    int32_t active;  // 0: the channel passes through (its sigma is on the FIR or identity branch)
    int32_t pad;
};

struct IirLaunch {
    int32_t seg_len;
    // 1: the transpose of the blur, for the adjoint of the render: both passes from a zero state, then a
    // correction at the far edge of each pass for the replicated edge state of the forward blur
    int32_t adjoint;
    IirChannel ch[3 * SPKB_MAX_COMPONENTS];  // [component * 3 + channel]
};

struct IirMixture {
    uint32_t ncomp;
    // 1: a plain blur, raw := G_0(src) with one component (weight, mix_a and mix_b unused); the column
    // pass stores the blurred lines as they are and never reads raw
    uint32_t plain;
    float weight[SPKB_MAX_COMPONENTS][3];
    float mix_a[3], mix_b[3];  // raw := mix_a raw + mix_b sum_k weight_k G_k(raw)
    IirLaunch rows, cols;
};

struct IirPlanes {
    float* p[SPKB_MAX_COMPONENTS];
};

size_t iir_rows_smem(uint32_t w);
size_t iir_cols_smem(uint32_t h);
int iir_row_seg_len(uint32_t w);  // segment length of the row and column passes for this frame
int iir_col_seg_len(uint32_t h);
bool iir_mixture_fits(uint32_t w, uint32_t h);  // both kernels' lines fit in shared memory

// raw := mix_a raw + mix_b sum_k weight_k G_k(src), every component recursive on every active channel
// (an inactive channel's lines pass through G_k unchanged); src is raw itself or, for a plain blur, any
// plane (raw := G_0(src)). tmp: ncomp planes for the row results; acc: one plane for the running sum
// (unused for one component).
void iir_mixture(const float* src, float* raw, float* const* tmp, float* acc, uint32_t w, uint32_t h,
                 const IirMixture& m, cudaStream_t s);

// Test hooks of the column pass's bounded TMA waits: the SM clocks a strip wait may take before it gives
// up (0: the full limit, about 2 s; process-wide), and the number of waits that gave up since the last
// call (read and reset on stream s, which is synchronised).
void set_iir_wait_limit(long long cycles);
uint32_t take_iir_waits_given_up(cudaStream_t s);

}  // namespace spkb::dev
