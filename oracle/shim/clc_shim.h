// clc_shim.h -- lets OpenCL C 1.x kernel source compile as C++17 for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY.  This header is part of the oracle: it is used to
// run the reference's own kernel files (src/*/*.cl) serially (or with OpenMP
// over work items) on the host so that the CUDA product can be checked against
// them.  Nothing in the product library includes it.
//
// Each work item sees its NDRange coordinates through a thread-local record
// that the fake OpenCL runtime (CL/cl.hpp in this directory) fills in before
// calling the kernel function.
#ifndef ORACLE_CLC_SHIM_H
#define ORACLE_CLC_SHIM_H

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <type_traits>

typedef unsigned int uint;

#define __kernel
#define __global
#define __local
#define __constant static const
#define KERNEL_PROGRAM 1

namespace clshim {
struct WorkItem {
    size_t gid[3];
    size_t gsize[3];
};
// Defined in cl_runtime.cpp; one record per host thread.
extern thread_local WorkItem g_wi;
}  // namespace clshim

static inline size_t get_global_id(uint d) { return clshim::g_wi.gid[d]; }
static inline size_t get_global_size(uint d) { return clshim::g_wi.gsize[d]; }
static inline size_t get_global_offset(uint) { return 0; }

static inline float as_float(uint x) {
    float f;
    std::memcpy(&f, &x, sizeof f);
    return f;
}

// OpenCL scalar select(a, b, c): c ? b : a.
template <class A, class B, class C>
static inline typename std::common_type<A, B>::type select(A a, B b, C c) {
    return c ? b : a;
}

#endif  // ORACLE_CLC_SHIM_H
