// Test infrastructure (oracle): the reference engine's kernels/probe.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "probe.metal"
REGISTER_KERNEL(spk_probe_fma);
REGISTER_KERNEL(spk_probe_philox);
