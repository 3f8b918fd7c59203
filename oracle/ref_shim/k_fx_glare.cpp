// Test infrastructure (oracle): the reference engine's kernels/fx_glare.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "fx_glare.metal"
REGISTER_KERNEL(spk_fx_glare_add);
