// Test infrastructure (oracle): the reference engine's kernels/session.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "session.metal"
REGISTER_KERNEL(spk_session_blur_v);
REGISTER_KERNEL(spk_session_blur_h);
REGISTER_KERNEL(spk_session_resample);
REGISTER_KERNEL(spk_session_copy_source);
