// rt_word.cuh -- word-parallel site arithmetic of the int8 models
// (dominoes, uniform lozenges): four sites of a colour-array row per 32-bit
// word.  Used by the single-walk word kernel (rt_word.cu) and the batched
// kernels (rt_batch.cu).
#pragma once

#include "rt_internal.h"
#include "rt_models.cuh"

namespace rtb {

// 0x01 in every byte of v equal to the same byte of pat (bytes < 0x80).
__device__ __forceinline__ uint32_t eq_bytes(uint32_t v, uint32_t pat) {
    const uint32_t x = v ^ pat;
    return (~(x + 0x7f7f7f7fu) >> 7) & 0x01010101u;
}

// 0x01 in byte b iff k_b < thr.
__device__ __forceinline__ uint32_t below4(const uint32_t (&k)[4], uint32_t thr) {
    return (uint32_t)(k[0] < thr) | ((uint32_t)(k[1] < thr) << 8) | ((uint32_t)(k[2] < thr) << 16) |
           ((uint32_t)(k[3] < thr) << 24);
}

__device__ __forceinline__ uint32_t lds(const unsigned char* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ void sts(unsigned char* p, uint32_t v) { *reinterpret_cast<uint32_t*>(p) = v; }

// Domino UpdateTiles (dominokernel.cl:22-31) for the four sites of a word:
// edge bits 1 up, 2 down, 4 towards j-1, 8 towards j+1 from the flipped array
// `src`; the neighbour towards j+1 shares the column in rows with
// p = (i + t) odd, towards j-1 in the others.
__device__ __forceinline__ uint32_t domino_refresh(const unsigned char* src, int off, int W, int p) {
    const uint32_t up = lds(src + off - W), dn = lds(src + off + W);
    const uint32_t l = lds(src + off - 4), c = lds(src + off), r = lds(src + off + 4);
    const uint32_t west = p ? c : __funnelshift_l(l, c, 8);
    const uint32_t east = p ? __funnelshift_r(c, r, 8) : c;
    return ((up & 0x02020202u) >> 1) | ((dn & 0x01010101u) << 1) | ((west & 0x08080808u) >> 1) |
           ((east & 0x04040404u) << 1);
}

// Lozenge UpdateTiles (lozengekernel.cl:36-54) for four sites: colour t+1
// keeps all but bits {2,4,32} and takes them from f[i-1][j+sa], f[i][j-sw],
// f[i+1][j]; colour t+2 keeps all but {1,8,16} and takes them from f[i-1][j],
// f[i][j+se], f[i+1][j-sa].  The bit fields never overlap, so the reference's
// sums are ORs.
__device__ __forceinline__ void lozenge_refresh(const unsigned char* f, int off, int W, uint32_t sh, uint32_t a_old,
                                                uint32_t b_old, uint32_t& na, uint32_t& nb) {
    const uint32_t u0 = lds(f + off - W), u1 = lds(f + off - W + 4);
    const uint32_t ml = lds(f + off - 4), m0 = lds(f + off), mr = lds(f + off + 4);
    const uint32_t dl = lds(f + off + W - 4), d0 = lds(f + off + W);
    const uint32_t sa = sh & 1u, sw = (sh >> 1) & 1u, se = (sh >> 2) & 1u;
    const uint32_t fu_sa = sa ? __funnelshift_r(u0, u1, 8) : u0;
    const uint32_t fw = sw ? __funnelshift_l(ml, m0, 8) : m0;
    const uint32_t fe = se ? __funnelshift_r(m0, mr, 8) : m0;
    const uint32_t fd_sa = sa ? __funnelshift_l(dl, d0, 8) : d0;
    na = (a_old & 0xd9d9d9d9u) | ((fu_sa & 0x10101010u) >> 3) | ((fw & 0x08080808u) >> 1) |
         ((d0 & 0x01010101u) << 5);
    nb = (b_old & 0xe6e6e6e6u) | ((u0 & 0x20202020u) >> 5) | ((fe & 0x04040404u) << 1) |
         ((fd_sa & 0x02020202u) << 3);
}

__device__ __forceinline__ uint32_t merge(uint32_t old, uint32_t nw, uint32_t mask) { return (old & ~mask) | (nw & mask); }

// Fixed facts of one word of the band: its byte offset in a colour plane,
// its colour-array row i, and two byte masks: `um` (0xff) marks the sites an
// Update refreshes (1 <= i <= N-2, 1 <= j <= width-2), `vm` (0x01) the sites
// that are Rotate positions.
struct WordInfo {
    int off;
    int cls;  // lozenges: i mod 3; dominoes: i mod 2
    uint32_t um;
    uint32_t vm;
};

template <int FAM>
struct WordModel {
    static constexpr bool DOM = FAM != FAM_LOZENGE8;
    static constexpr int NC = DOM ? 2 : 3;
    static constexpr int ROFF = DOM ? 1 : 0;
    static constexpr int COFF = DOM ? 1 : 0;
    __device__ static uint32_t written(uint32_t d) {
        if (ph_op(d) != OP_STEP) return 0u;
        return 1u << (DOM ? 1 - (int)ph_a(d) : (int)ph_a(d));
    }
};

// Per-phase decoded descriptor: which planes a word reads and writes.
struct WordPhase {
    bool step, upd, keep_a;
    int par;                // dominoes: parity t of the pending Update
    uint32_t shifts;        // lozenges: column shifts per row class (3 bits each)
    unsigned char* dst;     // dominoes: array written; lozenges: colour flipped (STEP)
    const unsigned char* src;  // flipped array whose neighbours are read (Update)
    unsigned char* pa;      // lozenges: colours t+1, t+2 of the Update
    unsigned char* pb;
};

__device__ __forceinline__ uint32_t lozenge_shift_table(int t) {
    uint32_t tab = 0;
#pragma unroll
    for (int rr = 0; rr < 3; ++rr) {
        const uint32_t sa = rr == (2 * t + 1) % 3, sw = rr == (2 * t + 2) % 3, se = rr == (2 * t) % 3;
        tab |= (sa | (sw << 1) | (se << 2)) << (3 * rr);
    }
    return tab;
}

// One phase on one word of one lattice; `lo` is the byte offset of the
// lattice's planes from those the phase descriptor points at.
// m0 / m1: per-byte draw masks (0x01) -- dominoes: k < thr[0]; lozenges:
// k < thr[0] (add a cube) and thr[0] <= k < thr[1] (remove one).
template <int FAM>
__device__ __forceinline__ void word_phase(const WordPhase& P, int lo, int W, const WordInfo& wi, uint32_t m0,
                                           uint32_t m1) {
    const int off = wi.off + lo;
    if (FAM != FAM_LOZENGE8) {
        uint32_t v = lds(P.dst + off);
        if (P.upd) v = merge(v, domino_refresh(P.src, off, W, (wi.cls ^ P.par) & 1), wi.um);
        if (P.step) {
            const uint32_t e3 = eq_bytes(v, 0x03030303u), e12 = eq_bytes(v, 0x0c0c0c0cu);
            uint32_t tog;
            if (FAM == FAM_DOMINO_HB)  // dominokernelCFTP.cl:19-28: k < 2^22 -> 12, else -> 3
                tog = (e3 & m0) | (e12 & ~m0);
            else  // dominokernel.cl:11-17: k < thr toggles 3 <-> 12
                tog = (e3 | e12) & m0;
            v ^= (tog & wi.vm) * 15u;
        }
        sts(P.dst + off, v);
    } else {
        if (P.step) {
            uint32_t v;
            if (P.upd) {
                const uint32_t ao = lds(P.pa + off), bo = lds(P.pb + off);
                uint32_t na, nb;
                lozenge_refresh(P.src, off, W, (P.shifts >> (3 * wi.cls)) & 7u, ao, bo, na, nb);
                na = merge(ao, na, wi.um);
                nb = merge(bo, nb, wi.um);
                if (P.keep_a) {
                    v = na;
                    sts(P.pb + off, nb);
                } else {
                    v = nb;
                    sts(P.pa + off, na);
                }
            } else {
                v = lds(P.dst + off);
            }
            // lozengekernel.cl:19-31: k < thr0 turns 25 into 38, thr0 <= k < thr1 turns 38 into 25.
            const uint32_t tog = (eq_bytes(v, 0x19191919u) & m0) | (eq_bytes(v, 0x26262626u) & m1);
            v ^= (tog & wi.vm) * 63u;
            sts(P.dst + off, v);
        } else {
            const uint32_t ao = lds(P.pa + off), bo = lds(P.pb + off);
            uint32_t na, nb;
            lozenge_refresh(P.src, off, W, (P.shifts >> (3 * wi.cls)) & 7u, ao, bo, na, nb);
            sts(P.pa + off, merge(ao, na, wi.um));
            sts(P.pb + off, merge(bo, nb, wi.um));
        }
    }
}

// 0x01 per byte of the bits set in mask, one bit per byte index.
__device__ __forceinline__ uint32_t lane_bytes(uint32_t bits) {
    return (bits & 1u) | ((bits & 2u) << 7) | ((bits & 4u) << 14) | ((bits & 8u) << 21);
}

// Decodes phase descriptor d for a lattice whose NC planes start at `lat`
// (`plane` bytes each); tabs = lozenge_shift_table(0..2).
template <int FAM>
__device__ __forceinline__ WordPhase word_phase_of(uint32_t d, unsigned char* lat, int plane, const uint32_t* tabs) {
    WordPhase P;
    const int op = (int)ph_op(d), ca = (int)ph_a(d), cb = (int)ph_b(d);
    P.step = op == (int)OP_STEP;
    P.upd = P.step ? (cb != (int)NO_COLOUR && cb != ca) : true;
    const int tt = P.step ? (P.upd ? cb : 0) : ca;
    if (FAM != FAM_LOZENGE8) {
        // Reference colour r flips array 1 - r, then refreshes array r from it.
        const int flip_arr = P.step ? 1 - ca : ca;
        P.dst = lat + flip_arr * plane;
        P.src = lat + (1 - flip_arr) * plane;
        P.par = tt & 1;
        P.keep_a = false;
        P.shifts = 0u;
        P.pa = P.pb = nullptr;
    } else {
        const int t1 = tt == 2 ? 0 : tt + 1, t2 = tt == 0 ? 2 : tt - 1;
        P.dst = lat + ca * plane;
        P.src = lat + tt * plane;
        P.pa = lat + t1 * plane;
        P.pb = lat + t2 * plane;
        P.keep_a = P.step && P.upd && t1 == ca;
        P.shifts = tt == 0 ? tabs[0] : tt == 1 ? tabs[1] : tabs[2];
        P.par = 0;
    }
    return P;
}

}  // namespace rtb
