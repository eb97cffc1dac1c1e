// rt_device.cuh -- device building blocks of the persistent walk kernel.
//
// The walk of one lattice runs as ONE cooperative launch.  Each CTA owns a
// band of rows of the "position grid" (the reference's Rotate NDRange), each
// thread a fixed set of positions, and each position keeps its TinyMT state in
// registers for the whole walk: the reference instead reads 28 B and writes
// 16 B of generator state per work item per colour step
// (src/TinyMT/tinymt32.clh:286-319).  Colour steps are separated by
// point-to-point waits on the two neighbouring CTAs' progress counters, not by
// kernel launches or a grid-wide barrier: a step only reads rows i-1..i+1.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rtb {

// ---------------------------------------------------------------------------
// Phase descriptors (one uint32 per phase, built on the host).
//   bits 0..7   op
//   bits 8..15  a   (colour rotated in this phase, or the last one for FINAL)
//   bits 16..23 b   (colour rotated in the previous phase; 0xff = none)
//   bit  24     the phase draws one number from every position's stream
// ---------------------------------------------------------------------------
enum : uint32_t {
    OP_STEP = 1,   // deferred update from colour b (if b != a), then flip colour a
    OP_FINAL = 2,  // update every other colour from colour a (end of walk)
    PH_DRAWS = 1u << 24,
    NO_COLOUR = 0xffu
};
__host__ __device__ inline uint32_t ph_op(uint32_t d) { return d & 0xffu; }
__host__ __device__ inline uint32_t ph_a(uint32_t d) { return (d >> 8) & 0xffu; }
__host__ __device__ inline uint32_t ph_b(uint32_t d) { return (d >> 16) & 0xffu; }
__host__ __device__ inline uint32_t make_phase(uint32_t op, uint32_t a, uint32_t b, bool draws) {
    return op | (a << 8) | (b << 16) | (draws ? PH_DRAWS : 0u);
}

// ---------------------------------------------------------------------------
// TinyMT32 (Saito & Matsumoto, 2011), the per-work-item generator of the
// reference (src/TinyMT/tinymt32.clh:39-203).  Written from the published
// algorithm: 127-bit state s0..s3, parameters mat1/mat2/tmat.
// ---------------------------------------------------------------------------
struct TinyState {
    uint32_t s0, s1, s2, s3;
};
struct TinyParams {
    uint32_t mat1, mat2, tmat;
};

__device__ __forceinline__ void tiny_advance(TinyState& s, const TinyParams& p) {
    uint32_t x = (s.s0 & 0x7fffffffu) ^ s.s1 ^ s.s2;
    uint32_t y = s.s3;
    x ^= x << 1;
    y ^= (y >> 1) ^ x;
    const uint32_t mask = 0u - (y & 1u);
    s.s0 = s.s1;
    s.s1 = s.s2 ^ (p.mat1 & mask);
    s.s2 = (x ^ (y << 10)) ^ (p.mat2 & mask);
    s.s3 = y;
}

__device__ __forceinline__ uint32_t tiny_output(const TinyState& s, const TinyParams& p) {
    const uint32_t t1 = s.s0 + (s.s2 >> 8);
    return (s.s3 ^ t1) ^ (p.tmat & (0u - (t1 & 1u)));
}

// One draw as the 23-bit integer k of single01() = k * 2^-23
// (tinymt32.clh:81-93, :125-129).  All acceptance tests compare k against an
// integer threshold computed on the host, which reproduces the reference's
// float / double comparisons exactly.
__device__ __forceinline__ uint32_t tiny_draw23(TinyState& s, const TinyParams& p) {
    tiny_advance(s, p);
    return tiny_output(s, p) >> 9;
}

__device__ __forceinline__ void tiny_seed(TinyState& s, const TinyParams& p, uint32_t seed) {
    uint32_t v0 = seed, v1 = p.mat1, v2 = p.mat2, v3 = p.tmat;
    // status[i & 3] ^= i + 1812433253 * (status[(i-1) & 3] ^ (status[(i-1) & 3] >> 30)), i = 1..7
    v1 ^= 1u + 1812433253u * (v0 ^ (v0 >> 30));
    v2 ^= 2u + 1812433253u * (v1 ^ (v1 >> 30));
    v3 ^= 3u + 1812433253u * (v2 ^ (v2 >> 30));
    v0 ^= 4u + 1812433253u * (v3 ^ (v3 >> 30));
    v1 ^= 5u + 1812433253u * (v0 ^ (v0 >> 30));
    v2 ^= 6u + 1812433253u * (v1 ^ (v1 >> 30));
    v3 ^= 7u + 1812433253u * (v2 ^ (v2 >> 30));
    if ((v0 & 0x7fffffffu) == 0u && v1 == 0u && v2 == 0u && v3 == 0u) {
        v0 = 'T';
        v1 = 'I';
        v2 = 'N';
        v3 = 'Y';
    }
    s.s0 = v0;
    s.s1 = v1;
    s.s2 = v2;
    s.s3 = v3;
#pragma unroll
    for (int i = 0; i < 8; ++i) tiny_advance(s, p);
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), written from the paper:
// 10 rounds of two 32x32->64 multiplies with the published round constants and
// Weyl key increments.  Used by the fast mode as a stateless generator.
// ---------------------------------------------------------------------------
__host__ __device__ inline void philox_round(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0,
                                             uint32_t k1) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
}

// All four output words of Philox4x32-10 for counter (c0..c3) and key (k0, k1).
__host__ __device__ inline uint4 philox4(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                         uint32_t k1) {
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        philox_round(c0, c1, c2, c3, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return make_uint4(c0, c1, c2, c3);
}

// Fast-mode draws.  The site (i, j) that a work item flips lies in the 32-bit
// word u = i * ceil(width/4) + j/4 of four consecutive sites of its colour
// array row (`width` sites per row); at step s (counted within the epoch) of
// chain `chain` it uses output word (j mod 4) of
// Philox4x32-10(counter = (u, s mod 2^32, s / 2^32, chain), key = epoch key),
// and its top 23 bits are the draw k, so the integer acceptance thresholds of
// the TinyMT mode apply unchanged.
__host__ __device__ inline uint32_t quad_word(const uint4& w, int lane) {
    return lane == 0 ? w.x : lane == 1 ? w.y : lane == 2 ? w.z : w.w;
}

// ---------------------------------------------------------------------------
// Lattice access.  Neighbour values written by other CTAs in the previous
// phase are read at L2 (ld.global.cg), never from a possibly stale L1 line.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ int ld_site(const T* p) {
    return (int)__ldcg(p);
}
template <>
__device__ __forceinline__ int ld_site<int8_t>(const int8_t* p) {
    return (int)(int8_t)__ldcg(reinterpret_cast<const signed char*>(p));
}
template <class T>
__device__ __forceinline__ void st_site(T* p, int v) {
    *p = (T)v;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

enum : int { ERR_TIMEOUT = 1, ERR_BADOP = 2 };

}  // namespace rtb
