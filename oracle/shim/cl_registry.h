// Kernel registration helpers for the fake OpenCL runtime (oracle only).
//
// TEST INFRASTRUCTURE ONLY.  A kernel translation unit includes one reference
// .cl file inside a namespace and registers each __kernel function under its
// OpenCL name; cl::make_kernel later finds it by (program, name).
#ifndef ORACLE_CL_REGISTRY_H
#define ORACLE_CL_REGISTRY_H

#include <CL/cl.hpp>

#include <initializer_list>
#include <tuple>
#include <type_traits>
#include <utility>

#include "clc_shim.h"

namespace clshim {

template <class T>
inline T arg_as(const Arg& a) {
    if constexpr (std::is_pointer<T>::value) {
        return reinterpret_cast<T>(a.ptr);
    } else {
        return static_cast<T>(a.ival);
    }
}

// Runs `body` once per work item of the NDRange with g_wi set.  Serial order
// is gid0 outermost, gid2 innermost.
template <class F>
inline void run_ndrange(const size_t* gs, int dims, F&& body) {
    const size_t g0 = gs[0], g1 = dims > 1 ? gs[1] : 1, g2 = dims > 2 ? gs[2] : 1;
    const long long total = static_cast<long long>(g0 * g1 * g2);
    const int nt = num_threads();
    if (nt <= 1) {
        for (size_t i0 = 0; i0 < g0; ++i0)
            for (size_t i1 = 0; i1 < g1; ++i1)
                for (size_t i2 = 0; i2 < g2; ++i2) {
                    g_wi = WorkItem{{i0, i1, i2}, {g0, g1, g2}};
                    body();
                }
        return;
    }
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long long k = 0; k < total; ++k) {
        const size_t i2 = static_cast<size_t>(k) % g2;
        const size_t r = static_cast<size_t>(k) / g2;
        g_wi = WorkItem{{r / g1, r % g1, i2}, {g0, g1, g2}};
        body();
    }
}

template <class... P, size_t... I>
inline Launcher make_launcher_impl(void (*fn)(P...), std::index_sequence<I...>) {
    return [fn](const std::vector<Arg>& a, const size_t* gs, int dims) {
        auto tup = std::make_tuple(arg_as<typename std::remove_cv<P>::type>(a.at(I))...);
        run_ndrange(gs, dims, [&]() { fn(std::get<I>(tup)...); });
    };
}

template <class... P>
inline Launcher make_launcher(void (*fn)(P...)) {
    return make_launcher_impl(fn, std::index_sequence_for<P...>{});
}

inline bool register_program(const char* program,
                             std::initializer_list<std::pair<const char*, Launcher> > kernels) {
    for (const auto& k : kernels) register_kernel(program, k.first, k.second);
    return true;
}

}  // namespace clshim

#endif  // ORACLE_CL_REGISTRY_H
