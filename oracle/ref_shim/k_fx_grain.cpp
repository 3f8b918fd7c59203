// Test infrastructure (oracle): the reference engine's kernels/fx_grain.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "fx_grain.metal"
REGISTER_KERNEL(spk_fx_grain_draw);
REGISTER_KERNEL(spk_fx_grain_lognormal);
REGISTER_KERNEL(spk_fx_grain_test_sampler);
