// Test infrastructure (oracle): the reference engine's kernels/fx_blur.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "fx_blur.metal"
REGISTER_KERNEL(spk_fx_blur_fir_v);
REGISTER_KERNEL(spk_fx_blur_fir_h);
REGISTER_KERNEL(spk_fx_blur_iir_h);
REGISTER_KERNEL(spk_fx_blur_iir_v);
REGISTER_KERNEL(spk_fx_blur_lincomb);
REGISTER_KERNEL(spk_fx_blur_affine);
REGISTER_KERNEL(spk_fx_blur_mul);
REGISTER_KERNEL(spk_fx_blur_copy);
