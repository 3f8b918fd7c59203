// Test infrastructure (oracle): the reference engine's kernels/fx_halation.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "fx_halation.metal"
REGISTER_KERNEL(spk_fx_halation_headroom);
REGISTER_KERNEL(spk_fx_halation_tent_down);
REGISTER_KERNEL(spk_fx_halation_up_mix);
