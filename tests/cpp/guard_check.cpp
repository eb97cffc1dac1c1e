// Host check of rt_guard.h: guarded() passes a status through, turns
// std::bad_alloc into RT_E_NOMEM and any other exception into RT_E_INVAL.
#include <cstdio>
#include <new>
#include <stdexcept>
#include <vector>

#include "rt_guard.h"

int main() {
    using rtb::guarded;
    int bad = 0;
    bad += guarded([] { return RT_OK; }) != RT_OK;
    bad += guarded([] { return RT_E_TIMEOUT; }) != RT_E_TIMEOUT;
    bad += guarded([]() -> rt_status { throw std::bad_alloc(); }) != RT_E_NOMEM;
    bad += guarded([]() -> rt_status { throw std::length_error("x"); }) != RT_E_INVAL;
    bad += guarded([]() -> rt_status { throw 7; }) != RT_E_INVAL;
    // an allocation the allocator cannot satisfy
    bad += guarded([]() -> rt_status {
        std::vector<char> v;
        v.reserve(v.max_size());
        return RT_OK;
    }) == RT_OK;
    std::printf(bad ? "FAIL %d\n" : "ok\n", bad);
    return bad ? 1 : 0;
}
