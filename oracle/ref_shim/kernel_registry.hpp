// Test infrastructure (oracle): runs the reference engine's Metal kernels, compiled as host C++, over
// their dispatch grid on the CPU with OpenMP.
//
// A kernel is registered by name with one line, REGISTER_KERNEL(spk_film_upsample). Its argument list
// is read from the function type: every parameter but the last is a buffer (pointer) or a by-value
// struct (reference) bound at the index of its position, exactly as the host's gpu::Arg list binds
// them; the last parameter is the grid position, `uint` for a 1-D dispatch or `uint2` for 2-D.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>

namespace spkref {

// slots[i]: the address of argument i (buffer contents + offset, or the by-value bytes).
using KernelThunk = void (*)(void* const* slots, uint32_t gx, uint32_t gy);

struct KernelInfo {
    KernelThunk run = nullptr;
    int dims = 1;
};

void register_kernel(const char* name, KernelThunk run, int dims);
const KernelInfo* find_kernel(const std::string& name);

template <class T>
inline T bind_slot(void* p) {
    if constexpr (std::is_pointer_v<T>) {
        return static_cast<T>(p);
    } else {
        static_assert(std::is_reference_v<T>, "kernel arguments are pointers or references");
        return *static_cast<std::remove_reference_t<T>*>(p);
    }
}

template <class F, F f>
struct Thunk;

template <class... A, void (*f)(A...)>
struct Thunk<void (*)(A...), f> {
    static constexpr size_t N = sizeof...(A);
    using Args = std::tuple<A...>;
    using Grid = std::tuple_element_t<N - 1, Args>;
    static constexpr int dims = std::is_same_v<std::decay_t<Grid>, uint32_t> ? 1 : 2;

    template <size_t... I>
    static void call(void* const* s, Grid g, std::index_sequence<I...>) {
        f(bind_slot<std::tuple_element_t<I, Args>>(s[I])..., g);
    }
    static void run(void* const* s, uint32_t gx, uint32_t gy) {
        if constexpr (dims == 1) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < int64_t(gx); ++i) call(s, Grid(uint32_t(i)), std::make_index_sequence<N - 1>{});
        } else {
#pragma omp parallel for schedule(static)
            for (int64_t y = 0; y < int64_t(gy); ++y)
                for (uint32_t x = 0; x < gx; ++x) call(s, Grid(x, uint32_t(y)), std::make_index_sequence<N - 1>{});
        }
    }
};

struct Registrar {
    Registrar(const char* name, KernelThunk run, int dims) { register_kernel(name, run, dims); }
};

}  // namespace spkref

#define REGISTER_KERNEL(fn)                                                                                  \
    static spkref::Registrar reg_##fn(#fn, &spkref::Thunk<decltype(&fn), &fn>::run,                          \
                                      spkref::Thunk<decltype(&fn), &fn>::dims)
