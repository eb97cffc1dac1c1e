// rt_exchange.cuh -- halo-row exchange between the CTAs of one walk.
#pragma once

#include "rt_models.cuh"

namespace rtb {

// ---------------------------------------------------------------------------
// Halo exchange.  After each flip phase a CTA publishes the first and last
// row of its band (of the colour it just flipped) into a slot of global
// memory; every 64-bit slot word carries 32 bits of lattice data and the
// phase tag (phase + 1), so a neighbour knows the row is complete by polling
// the words themselves -- no separate flag, no memory fence on the critical
// path.  Slots are double-buffered by phase parity; a CTA enters phase p only
// after both neighbours finished phase p-1, so a slot is never overwritten
// before it was read.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long* slot(const WalkArgs& a, int cta, int side, int parity, int lat,
                                                   int k) {
    return a.xbuf + (((((size_t)cta * 2 + side) * 2 + parity) * a.nlat + lat) * a.xslots + k) * a.xwords;
}

// Index of the k-th set bit of mask (k < popc(mask)).
__device__ __forceinline__ int nth_bit(uint32_t mask, int k) {
    for (int i = 0; i < k; ++i) mask &= mask - 1;
    return __ffs(mask) - 1;
}

template <class T>
__device__ __forceinline__ uint32_t pack_word(const T* row, int w) {
    if (sizeof(T) == 1) return reinterpret_cast<const uint32_t*>(row)[w];
    return (uint32_t)row[w];
}
template <class T>
__device__ __forceinline__ void unpack_word(T* row, int w, uint32_t v) {
    if (sizeof(T) == 1)
        reinterpret_cast<uint32_t*>(row)[w] = v;
    else
        row[w] = (T)v;
}

// Waits for one tagged word; returns false on timeout (a.timeout_ns from the
// first check of this wait's clock) or when another CTA already reported an
// error.  The clock starts at this wait, so a walk may run for any length of
// time; only a single wait is bounded.
__device__ __forceinline__ bool wait_word(const WalkArgs& a, const unsigned long long* p, uint32_t tag,
                                          uint32_t* out) {
    unsigned spins = 0;
    uint64_t t0 = 0;
    for (;;) {
        const unsigned long long x = ld_relaxed64(p);
        if ((uint32_t)(x >> 32) == tag) {
            *out = (uint32_t)x;
            return true;
        }
        if ((++spins & 63u) == 0u) {
            if (*(volatile int*)a.err) return false;
            const uint64_t now = global_ns();
            if (t0 == 0) {
                t0 = now;
            } else if (now - t0 > a.timeout_ns) {
                atomicOr(a.err, ERR_TIMEOUT);
                return false;
            }
        }
    }
}

}  // namespace rtb
