// Test infrastructure (oracle): the reference engine's kernels/print.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "print.metal"
REGISTER_KERNEL(spk_print_spectral);
REGISTER_KERNEL(spk_print_gain);
REGISTER_KERNEL(spk_print_paper);
REGISTER_KERNEL(spk_print_levels);
REGISTER_KERNEL(spk_print_matrix);
REGISTER_KERNEL(spk_print_gamut);
REGISTER_KERNEL(spk_print_edr);
REGISTER_KERNEL(spk_print_encode);
REGISTER_KERNEL(spk_print_lut);
