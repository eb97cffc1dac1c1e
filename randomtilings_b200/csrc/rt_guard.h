// rt_guard.h -- keeps C++ exceptions from crossing the C ABI.
//
// The exported functions of the host-side files run their bodies through
// guarded(): an allocation that fails (std::bad_alloc, e.g. a buffer sized
// from a very large argument) returns RT_E_NOMEM, and anything else thrown
// returns RT_E_INVAL, instead of terminating the caller's process.
#pragma once

#include <new>

#include "../../include/rt_b200.h"

namespace rtb {

template <class F>
rt_status guarded(F&& f) noexcept {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return RT_E_NOMEM;
    } catch (...) {
        return RT_E_INVAL;
    }
}

}  // namespace rtb
