// The per-channel plan of one Gaussian blur (the reference's branch rule, src/fx/gaussian.hpp:6-15):
// sigma <= 0 identity, sigma < 3 FIR with R = floor(3 sigma + 0.5), otherwise the recursive filter.
// Kept free of the host set-up headers so that CUDA translation units can include it.
#pragma once

#include <cuda_runtime.h>

#include "../kernel_args.h"

namespace spkb {

enum BlurBranchCode { BLUR_IDENTITY = 0, BLUR_FIR = 1, BLUR_IIR = 2 };

int blur_branch_code(double sigma);
// FIR taps of the non-recursive channels (a delta on the others), common radius
FirTaps blur_fir_taps(const double sigma[3], const bool iir[3]);
// recursive coefficients of the channels with iir[c]
IirCoefs blur_iir_coefs(const double sigma[3], const bool iir[3]);
// dst := G(src) by the block-parallel recursive kernels (src == dst allowed): the channels with iir[c]
// blurred at sigma[c], the others passed through unchanged; tmp: one plane of scratch. Launches nothing
// and returns false when a plane's base is not 16-byte aligned or the frame's lines do not fit in shared
// memory. Allocates nothing.
bool blur_iir_block(const float* src, float* dst, float* tmp, uint32_t w, uint32_t h, const double sigma[3],
                    const bool iir[3], cudaStream_t s);

}  // namespace spkb
