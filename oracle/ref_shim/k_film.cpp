// Test infrastructure (oracle): the reference engine's kernels/film.metal, compiled as host C++ and registered
// for the CPU dispatcher. The kernel source is read where it lies; nothing of it is copied here.
#include "kernel_registry.hpp"
#include "film.metal"
REGISTER_KERNEL(spk_film_decode);
REGISTER_KERNEL(spk_film_geometry);
REGISTER_KERNEL(spk_film_scale);
REGISTER_KERNEL(spk_film_upsample);
REGISTER_KERNEL(spk_film_boost);
REGISTER_KERNEL(spk_film_log);
REGISTER_KERNEL(spk_film_curves);
REGISTER_KERNEL(spk_film_coupler_source);
REGISTER_KERNEL(spk_film_coupler_apply);
