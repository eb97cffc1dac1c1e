// rt_tdplane.cuh -- the triangle-dimer phase ops on bit planes.
//
// The eight state arrays of TriDimerRule (rt_tridimer.cuh) hold small
// integers: the lozenge arrays H, L, R four bits, the triangle arrays U, D
// three base-4 digits (six bits), the butterfly arrays BH, BL, BR four base-4
// digits and a centre bit (nine bits).  Here every bit of every array is a
// plane of its own, 32 sites of a row per 32-bit word, 51 planes in all, and
// each phase op is written as boolean algebra on the words: one work item
// updates 32 sites of a row at once.  A neighbour at column j +- 1 is a
// funnel shift of two adjacent words.  Sums of weighted conditions (the
// digits a + 2 b + 3 c of the reference's rules) use a bit-sliced ripple
// adder, so every value is the one the integer rule computes, modulo the
// array's width (states reached from a valid tiling never exceed it).
//
// Sites outside an op's mask keep their bits; within one phase no op reads a
// site it writes (the reference's parallel kernels rely on the same), so the
// new words are functions of the old state alone.  The functions compile for
// the host too, where the tests check each op against TriDimerRule.
#pragma once

#include <stdint.h>

#include "rt_tdops.h"

#ifdef __CUDACC__
#define TDP_HD __host__ __device__ __forceinline__
#else
#define TDP_HD inline
#endif

namespace rtb {
namespace tdp {

constexpr int kPlanes = 51;

// First plane and bit count of array `arr` (0 H, 1 L, 2 R, 3 U, 4 D, 5 BH, 6 BL, 7 BR).
TDP_HD constexpr int plane_of(int arr) { return arr < 3 ? 4 * arr : arr < 5 ? 12 + 6 * (arr - 3) : 24 + 9 * (arr - 5); }
TDP_HD constexpr int bits_of(int arr) { return arr < 3 ? 4 : arr < 5 ? 6 : 9; }

// The planes of one chain (or one band of it) and the work item (array row
// i, word c covering columns 32 c .. 32 c + 31).  Layout: plane-major, then
// rows (row 0 = array row row0), then words; the word before a row's first
// word and the word after its last one read as zero (the columns outside
// the array), e.g. rows of wb + 1 words whose last word stays zero, after
// one zero word.
struct View {
    uint32_t* p;  // plane 0, row 0, word 0
    int ps, rs;   // plane and row strides in words
    int row0;
    int i, c;
    TDP_HD uint32_t* word(int plane, int di) const { return p + plane * ps + (i - row0 + di) * rs + c; }
    // Plane `bit` of array `arr` at row i + di, columns shifted by dj (-1, 0, +1):
    // lane l holds the site (i + di, 32 c + l + dj).
    TDP_HD uint32_t ld(int arr, int bit, int di, int dj) const {
        const uint32_t* q = word(plane_of(arr) + bit, di);
        if (dj == 0) return q[0];
        if (dj > 0) return (q[0] >> 1) | (q[1] << 31);
        return (q[0] << 1) | (q[-1] >> 31);
    }
    TDP_HD void st(int arr, int bit, uint32_t v, uint32_t m) const {
        uint32_t* q = word(plane_of(arr) + bit, 0);
        *q = (*q & ~m) | (v & m);
    }
};

// ---- lane masks -------------------------------------------------------------
TDP_HD int mod3(int x) { return ((x % 3) + 3) % 3; }
// lanes of word c whose column j = 32 c + l has j mod 2 == r
TDP_HD uint32_t col_par(int r) { return (r & 1) ? 0xAAAAAAAAu : 0x55555555u; }
// lanes of word c whose column has j mod 3 == r (32 = 2 mod 3)
TDP_HD uint32_t col_mod3(int r, int c) {
    const int k = mod3(r - 2 * c);
    return k == 0 ? 0x49249249u : k == 1 ? 0x92492492u : 0x24924924u;
}
// lanes of word c whose column lies in [lo, hi]
TDP_HD uint32_t col_range(int c, int lo, int hi) {
    int a = lo - 32 * c, b = hi - 32 * c;
    if (b < 0 || a > 31 || a > b) return 0u;
    a = a < 0 ? 0 : a;
    b = b > 31 ? 31 : b;
    const uint32_t upto = b >= 31 ? 0xFFFFFFFFu : ((1u << (b + 1)) - 1u);
    const uint32_t below = (1u << a) - 1u;
    return upto & ~below;
}
TDP_HD uint32_t all_if(bool x) { return x ? 0xFFFFFFFFu : 0u; }

// ---- bit-sliced small integers -------------------------------------------------
// acc (n bits) += x (nx bits) << off, modulo 2^n.
template <int N>
TDP_HD void add_at(uint32_t (&acc)[N], const uint32_t* x, int nx, int off) {
    uint32_t carry = 0u;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (k < off) continue;
        const uint32_t xb = (k - off) < nx ? x[k - off] : 0u;
        const uint32_t a = acc[k];
        acc[k] = a ^ xb ^ carry;
        carry = (a & xb) | (carry & (a ^ xb));
    }
}
// w1 a + w2 b + w3 c for 0/1 lanes a, b, c and weights 0..3: three bits.
TDP_HD void wsum(uint32_t (&out)[3], int w1, uint32_t a, int w2, uint32_t b, int w3, uint32_t c) {
    out[0] = out[1] = out[2] = 0u;
    const uint32_t xa[2] = {(w1 & 1) ? a : 0u, (w1 & 2) ? a : 0u};
    const uint32_t xb[2] = {(w2 & 1) ? b : 0u, (w2 & 2) ? b : 0u};
    const uint32_t xc[2] = {(w3 & 1) ? c : 0u, (w3 & 2) ? c : 0u};
    add_at(out, xa, 2, 0);
    add_at(out, xb, 2, 0);
    add_at(out, xc, 2, 0);
}
// Lanes where the base-4 digit (lo, hi) equals v.
TDP_HD uint32_t deq(uint32_t lo, uint32_t hi, int v) {
    return ((v & 1) ? lo : ~lo) & ((v & 2) ? hi : ~hi);
}
// t1 + 4 t4 + 16 t16 + 64 t64 + 256 c (each t three bits) into nine planes.
TDP_HD void pack(uint32_t (&out)[9], const uint32_t (&t1)[3], const uint32_t (&t4)[3], const uint32_t (&t16)[3],
                 const uint32_t (&t64)[3], uint32_t c) {
#pragma unroll
    for (int k = 0; k < 9; ++k) out[k] = 0u;
    add_at(out, t1, 3, 0);
    add_at(out, t4, 3, 2);
    add_at(out, t16, 3, 4);
    add_at(out, t64, 3, 6);
    const uint32_t cc[1] = {c};
    add_at(out, cc, 1, 8);
}
// a digit (lo, hi) as a three-bit number
TDP_HD void dig3(uint32_t (&out)[3], uint32_t lo, uint32_t hi) {
    out[0] = lo;
    out[1] = hi;
    out[2] = 0u;
}
// lane-wise select: m ? x : y
TDP_HD void sel3(uint32_t (&out)[3], uint32_t m, const uint32_t (&x)[3], const uint32_t (&y)[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = (x[k] & m) | (y[k] & ~m);
}
TDP_HD void const3(uint32_t (&out)[3], int v) {
    out[0] = (v & 1) ? 0xFFFFFFFFu : 0u;
    out[1] = (v & 2) ? 0xFFFFFFFFu : 0u;
    out[2] = (v & 4) ? 0xFFFFFFFFu : 0u;
}


// ---- values built from the lozenge arrays ---------------------------------------
// Butterfly state of orientation `which` from the lozenges
// (UpdateButterflys{H,L,R}FromLozenge, triangledimerkernel.cl:118-189).
TDP_HD void bfly_from_loz(uint32_t (&out)[9], const View& v, int which) {
    uint32_t t1[3], t4[3], t16[3], t64[3], c;
    if (which == 0) {
        c = v.ld(1, 2, -1, 1);
        wsum(t1, 1, v.ld(2, 3, -1, 0), 2, v.ld(2, 0, -1, 0), 3, v.ld(0, 0, 0, 0));
        wsum(t4, 1, v.ld(1, 0, -1, 1), 2, v.ld(1, 1, -1, 1), 3, v.ld(0, 1, 0, 0));
        wsum(t16, 1, v.ld(2, 1, 0, 0), 2, v.ld(2, 2, 0, 0), 3, v.ld(0, 2, 0, 0));
        wsum(t64, 1, v.ld(1, 2, 0, 0), 2, v.ld(1, 3, 0, 0), 3, v.ld(0, 3, 0, 0));
    } else if (which == 1) {
        c = v.ld(2, 3, 0, 0);
        wsum(t1, 1, v.ld(0, 0, 0, 0), 2, v.ld(0, 1, 0, 0), 3, v.ld(1, 0, 0, 0));
        wsum(t4, 1, v.ld(2, 1, 0, 0), 2, v.ld(2, 2, 0, 0), 3, v.ld(1, 1, 0, 0));
        wsum(t16, 1, v.ld(0, 2, 1, -1), 2, v.ld(0, 3, 1, -1), 3, v.ld(1, 2, 0, 0));
        wsum(t64, 1, v.ld(2, 3, 0, -1), 2, v.ld(2, 0, 0, -1), 3, v.ld(1, 3, 0, 0));
    } else {
        c = v.ld(1, 3, 0, 1);
        wsum(t1, 1, v.ld(0, 0, 0, 0), 2, v.ld(0, 1, 0, 0), 3, v.ld(2, 0, 0, 0));
        wsum(t4, 1, v.ld(1, 0, 0, 1), 2, v.ld(1, 1, 0, 1), 3, v.ld(2, 1, 0, 0));
        wsum(t16, 1, v.ld(0, 2, 1, 0), 2, v.ld(0, 3, 1, 0), 3, v.ld(2, 2, 0, 0));
        wsum(t64, 1, v.ld(1, 2, 0, 0), 2, v.ld(1, 3, 0, 0), 3, v.ld(2, 3, 0, 0));
    }
    pack(out, t1, t4, t16, t64, c);
}

// Up-triangle state from the lozenges (UpdateTriangleUFromLozenges, :96-116).
TDP_HD void up_from_loz(uint32_t (&out)[6], const View& v) {
    uint32_t x[3], y[3], z[3];
    wsum(x, 1, v.ld(1, 0, 0, 0), 2, v.ld(0, 3, 0, 0), 3, v.ld(0, 0, 1, 0));
    wsum(y, 1, v.ld(1, 0, 0, 1), 2, v.ld(0, 1, 1, 0), 3, v.ld(1, 1, 0, 1));
    wsum(z, 1, v.ld(1, 2, 0, 1), 2, v.ld(0, 3, 1, 0), 3, v.ld(0, 2, 1, 0));
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = 0u;
    add_at(out, x, 3, 0);
    add_at(out, y, 3, 2);
    add_at(out, z, 3, 4);
}

// TriDimerRule::tri_digit of the triangle value at (di, dj) of array arr.
TDP_HD void tri_digit(uint32_t (&out)[3], const View& v, int arr, int di, int dj) {
    const uint32_t A = v.ld(arr, 4, di, dj) & ~v.ld(arr, 5, di, dj);  // (x & 48) == 16
    const uint32_t B = v.ld(arr, 0, di, dj) & v.ld(arr, 1, di, dj);   // (x & 3) == 3
    const uint32_t C = ~v.ld(arr, 2, di, dj) & v.ld(arr, 3, di, dj);  // (x & 12) == 8
    wsum(out, 1, A, 2, B, 3, C);
}

// ---- lane classes -----------------------------------------------------------------
// ((1 - (t & 1)) i + ((1 + t) / 2) j) mod 2 == r
TDP_HD uint32_t cls2(int t, int i, int r) {
    return t == 0 ? all_if((i & 1) == (r & 1)) : t == 1 ? col_par(r) : col_par((r - i) & 1);
}
// (j + 2 i) mod 3 == r
TDP_HD uint32_t cls3(int i, int c, int r) { return col_mod3(mod3(r - 2 * i), c); }
// TriDimerRule::slice(t, i, j) == r
TDP_HD uint32_t slice3(int t, int i, int c, int r) {
    return t == 0 ? all_if(mod3(i) == r) : t == 1 ? col_mod3(r, c) : col_mod3(mod3(r - i), c);
}
// TriDimerRule::bpar(t, i, j) == r
TDP_HD uint32_t bpar2(int t, int i, int r) { return t == 1 ? all_if((i & 1) == (r & 1)) : col_par(r); }

// digit k of a butterfly value at (di, dj): (lo, hi)
struct Dig {
    uint32_t lo, hi;
};
TDP_HD Dig bdig(const View& v, int arr, int k, int di, int dj) { return {v.ld(arr, 2 * k, di, dj), v.ld(arr, 2 * k + 1, di, dj)}; }
TDP_HD void d3(uint32_t (&out)[3], Dig d) { dig3(out, d.lo, d.hi); }
TDP_HD void d3(uint32_t (&out)[3], uint32_t lo, uint32_t hi) { dig3(out, lo, hi); }

// ---- the ops ------------------------------------------------------------------------
// One 32-site word of phase (OP, a, b) at the view's row and word.  T >= 0
// / B >= 0 fix a / b at compile time.  m: array side; width: columns in
// use; draw: lanes whose draw k is below 2^22 (drawing ops only).
template <uint32_t OP, int T = -1, int B = -1>
TDP_HD void word_op(const View& v, uint32_t a_, uint32_t b_, int m, int width, uint32_t draw) {
    const int t = T >= 0 ? T : (int)a_;
    const uint32_t bb = B >= 0 ? (uint32_t)B : b_;
    const int i = v.i, c = v.c;
    const uint32_t VAL = col_range(c, 0, width - 1);
    const uint32_t INT = (i >= 1 && i <= m - 2) ? col_range(c, 1, m - 2) : 0u;
    switch (OP) {
        case TD_ROT_LOZ: {  // :4-22
            uint32_t x[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) x[k] = v.ld(t, k, 0, 0);
            const uint32_t eq5 = x[0] & ~x[1] & x[2] & ~x[3], eq10 = ~x[0] & x[1] & ~x[2] & x[3];
            const uint32_t F = cls2(t, i, (int)bb) & draw & VAL & (eq5 | eq10);
#pragma unroll
            for (int k = 0; k < 4; ++k) v.st(t, k, ~x[k], F);
            break;
        }
        case TD_LOZ_FLIPPED: {  // :24-33
            const uint32_t M = INT & ~cls2(t, i, (int)bb);
            const int dj = t & 1, di = (2 - t) / 2;
            const uint32_t n0 = v.ld(t, 2, -1, dj), n1 = v.ld(t, 3, -di, 1), n2 = v.ld(t, 0, 1, -dj),
                           n3 = v.ld(t, 1, di, -1);
            v.st(t, 0, n0, M);
            v.st(t, 1, n1, M);
            v.st(t, 2, n2, M);
            v.st(t, 3, n3, M);
            break;
        }
        case TD_LOZ_OTHER: {  // :35-78
            const uint32_t M = INT;
            if (t == 0) {
                const uint32_t l1 = v.ld(0, 0, 1, 0), l3 = v.ld(0, 0, 1, -1), r1 = v.ld(0, 1, 1, 0), r3 = v.ld(0, 3, 0, 0);
                v.st(1, 1, l1, M);
                v.st(1, 3, l3, M);
                v.st(2, 1, r1, M);
                v.st(2, 3, r3, M);
            } else if (t == 1) {
                const uint32_t r0 = v.ld(1, 0, 0, 0), r2 = v.ld(1, 0, 1, 0), h0 = v.ld(1, 1, -1, 0), h2 = v.ld(1, 1, 0, 0);
                v.st(2, 0, r0, M);
                v.st(2, 2, r2, M);
                v.st(0, 0, h0, M);
                v.st(0, 2, h2, M);
            } else {
                const uint32_t h1 = v.ld(2, 1, -1, 0), h3 = v.ld(2, 1, 0, -1), l0 = v.ld(2, 0, 0, 0), l2 = v.ld(2, 2, 0, -1);
                v.st(0, 1, h1, M);
                v.st(0, 3, h3, M);
                v.st(1, 0, l0, M);
                v.st(1, 2, l2, M);
            }
            break;
        }
        case TD_UP_FROM_LOZ: {
            uint32_t u[6];
            up_from_loz(u, v);
#pragma unroll
            for (int k = 0; k < 6; ++k) v.st(3, k, u[k], INT);
            break;
        }
        case TD_TRI_OTHER: {  // :255-275, then :118-189 for the butterflies in b
            const int src = t == 0 ? 3 : 4, dst = t == 0 ? 4 : 3, p = t == 0 ? -1 : 1;
            uint32_t d0[3], d1[3], d2[3], tv[6] = {0u, 0u, 0u, 0u, 0u, 0u};
            tri_digit(d0, v, src, 0, -1 + t);
            tri_digit(d1, v, src, 0, t);
            tri_digit(d2, v, src, p, 0);
            add_at(tv, d0, 3, 0);
            add_at(tv, d1, 3, 2);
            add_at(tv, d2, 3, 4);
            uint32_t bv[3][9];
#pragma unroll
            for (int w = 0; w < 3; ++w)
                if (bb & (1u << w)) bfly_from_loz(bv[w], v, w);
#pragma unroll
            for (int k = 0; k < 6; ++k) v.st(dst, k, tv[k], INT);
#pragma unroll
            for (int w = 0; w < 3; ++w)
                if (bb & (1u << w)) {
#pragma unroll
                    for (int k = 0; k < 9; ++k) v.st(5 + w, k, bv[w][k], INT);
                }
            break;
        }
        case TD_ROT_TRI: {  // :191-211
            const int arr = t == 1 ? 4 : 3;
            uint32_t x[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) x[k] = v.ld(arr, k, 0, 0);
            const uint32_t eq45 = x[0] & ~x[1] & x[2] & x[3] & ~x[4] & x[5];
            const uint32_t eq54 = ~x[0] & x[1] & x[2] & ~x[3] & x[4] & x[5];
            const uint32_t F = cls3(i, c, (int)bb) & draw & VAL & (eq45 | eq54);
            v.st(arr, 0, ~x[0], F);
            v.st(arr, 1, ~x[1], F);
            v.st(arr, 3, ~x[3], F);
            v.st(arr, 4, ~x[4], F);
            break;
        }
        case TD_TRI_FLIPPED: {  // :213-253
            const int arr = t == 1 ? 4 : 3;
            const uint32_t M1 = INT & cls3(i, c, ((int)bb + 1) % 3), M2 = INT & cls3(i, c, ((int)bb + 2) % 3);
            uint32_t vp[6], vq[6];
            // p: digit 1 of (0,-1), digit 2 of (-1,+1) [t = 1: (+1,0)], digit 0 of (+1,0) [t = 1: (-1,+1)]
            const int ai = t == 0 ? -1 : 1, aj = t == 0 ? 1 : 0, ci = t == 0 ? 1 : -1, cj = t == 0 ? 0 : 1;
            vp[0] = v.ld(arr, 2, 0, -1);
            vp[1] = v.ld(arr, 3, 0, -1);
            vp[2] = v.ld(arr, 4, ai, aj);
            vp[3] = v.ld(arr, 5, ai, aj);
            vp[4] = v.ld(arr, 0, ci, cj);
            vp[5] = v.ld(arr, 1, ci, cj);
            // not p: digit 2 of (-1,0) [t = 1: (+1,-1)], digit 0 of (0,+1), digit 1 of (+1,-1) [t = 1: (-1,0)]
            const int ei = t == 0 ? -1 : 1, ej = t == 0 ? 0 : -1, gi = t == 0 ? 1 : -1, gj = t == 0 ? -1 : 0;
            vq[0] = v.ld(arr, 4, ei, ej);
            vq[1] = v.ld(arr, 5, ei, ej);
            vq[2] = v.ld(arr, 0, 0, 1);
            vq[3] = v.ld(arr, 1, 0, 1);
            vq[4] = v.ld(arr, 2, gi, gj);
            vq[5] = v.ld(arr, 3, gi, gj);
#pragma unroll
            for (int k = 0; k < 6; ++k) v.st(arr, k, (vp[k] & M1) | (vq[k] & M2), M1 | M2);
            break;
        }
        case TD_LOZ_FROM_TRI: {  // :277-329
            uint32_t dd[6], uh4, uh5, ul2, ul3, ur0, ur1;
#pragma unroll
            for (int k = 0; k < 6; ++k) dd[k] = v.ld(4, k, 0, 0);
            uh4 = v.ld(3, 4, -1, 0);
            uh5 = v.ld(3, 5, -1, 0);
            ul2 = v.ld(3, 2, 0, -1);
            ul3 = v.ld(3, 3, 0, -1);
            ur0 = v.ld(3, 0, 0, 0);
            ur1 = v.ld(3, 1, 0, 0);
            const uint32_t M = INT;
            v.st(0, 0, ~dd[4] & dd[5], M);
            v.st(0, 1, dd[4] & dd[5], M);
            v.st(0, 2, uh4 & uh5, M);
            v.st(0, 3, ~uh4 & uh5, M);
            v.st(1, 0, ul2 & ~ul3, M);
            v.st(1, 1, ul2 & ul3, M);
            v.st(1, 2, dd[0] & ~dd[1], M);
            v.st(1, 3, ~dd[0] & dd[1], M);
            v.st(2, 0, ur0 & ~ur1, M);
            v.st(2, 1, dd[2] & dd[3], M);
            v.st(2, 2, dd[2] & ~dd[3], M);
            v.st(2, 3, ~ur0 & ur1, M);
            break;
        }
        case TD_BFLY_FROM_LOZ: {
            uint32_t bv[3][9], uv[6];
#pragma unroll
            for (int w = 0; w < 3; ++w)
                if (bb & (1u << w)) bfly_from_loz(bv[w], v, w);
            if (t) up_from_loz(uv, v);  // a = 1: also U from the lozenges
#pragma unroll
            for (int w = 0; w < 3; ++w)
                if (bb & (1u << w)) {
#pragma unroll
                    for (int k = 0; k < 9; ++k) v.st(5 + w, k, bv[w][k], INT);
                }
            if (t) {
#pragma unroll
                for (int k = 0; k < 6; ++k) v.st(3, k, uv[k], INT);
            }
            break;
        }
        case TD_ROT_BFLY: {  // :331-353
            const int p1 = (int)(bb & 3), p2 = (int)(bb >> 2);
            const uint32_t cond = t == 0   ? all_if(mod3(i) == p1) & col_par(p2)
                                  : t == 1 ? col_mod3(p1, c) & all_if((i & 1) == p2)
                                           : col_mod3(mod3(p1 - i), c) & col_par(p2);
            uint32_t x[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) x[k] = v.ld(5 + t, k, 0, 0);
            // 170 = bits 1, 3, 5, 7; 85 = bits 0, 2, 4, 6; the centre bit clear in both
            const uint32_t odd = x[1] & x[3] & x[5] & x[7], even = x[0] & x[2] & x[4] & x[6];
            const uint32_t nodd = ~x[1] & ~x[3] & ~x[5] & ~x[7], neven = ~x[0] & ~x[2] & ~x[4] & ~x[6];
            const uint32_t F = cond & draw & VAL & ~x[8] & ((odd & neven) | (even & nodd));
#pragma unroll
            for (int k = 0; k < 8; ++k) v.st(5 + t, k, ~x[k], F);
            break;
        }
        case TD_BFLY_SAME: {  // UpdateButterflysFlipped{H,L,R}1
            const int p1 = (int)(bb & 3), p2 = (int)(bb >> 2);
            const int arr = 5 + t;
            const uint32_t M = INT & slice3(t, i, c, p1) & ~bpar2(t, i, p2);
            Dig t1, t4, t16, t64;
            // cyc_up (0,1,2,3 -> 0,2,3,1): (lo, hi) -> (hi, hi ^ lo); cyc_dn (-> 0,3,1,2): -> (hi ^ lo, lo)
            auto up = [](Dig d) { return Dig{d.hi, d.hi ^ d.lo}; };
            auto dn = [](Dig d) { return Dig{d.hi ^ d.lo, d.lo}; };
            if (t == 2) {
                t1 = dn(bdig(v, arr, 3, -1, 1));
                t4 = up(bdig(v, arr, 2, -1, 1));
                t16 = dn(bdig(v, arr, 1, 1, -1));
                t64 = up(bdig(v, arr, 0, 1, -1));
            } else {
                const int ui = t == 0 ? 0 : -1, uj = t == 0 ? -1 : 0, vi = t == 0 ? 0 : 1, vj = t == 0 ? 1 : 0;
                t1 = up(bdig(v, arr, 1, ui, uj));
                t4 = dn(bdig(v, arr, 0, vi, vj));
                t16 = up(bdig(v, arr, 3, vi, vj));
                t64 = dn(bdig(v, arr, 2, ui, uj));
            }
            const uint32_t out[8] = {t1.lo, t1.hi, t4.lo, t4.hi, t16.lo, t16.hi, t64.lo, t64.hi};
#pragma unroll
            for (int k = 0; k < 8; ++k) v.st(arr, k, out[k], M);
            break;
        }
        case TD_BFLY_21: {
            const int p1 = (int)bb;
            const int want = t == 0 ? (p1 + 1) % 3 : (p1 + 2) % 3;
            const int arr = 5 + t;
            const uint32_t M = INT & slice3(t, i, c, want);
            const Dig f0 = bdig(v, arr, 0, 0, 0), f1 = bdig(v, arr, 1, 0, 0), f2 = bdig(v, arr, 2, 0, 0),
                      f3 = bdig(v, arr, 3, 0, 0);
            uint32_t t1[3], t4[3], t16[3], t64[3], cc, alt[3], k3[3];
            if (t == 2) {
                const Dig e0 = bdig(v, arr, 0, 0, 1), e3 = bdig(v, arr, 3, 0, 1), s0 = bdig(v, arr, 0, 1, 0),
                          s3 = bdig(v, arr, 3, 1, 0);
                cc = deq(s0.lo, s0.hi, 1);
                d3(t1, f0);
                wsum(alt, 1, deq(e0.lo, e0.hi, 3), 3, deq(e3.lo, e3.hi, 3), 0, 0u);
                const3(k3, 2);
                sel3(t4, deq(f1.lo, f1.hi, 2), k3, alt);
                wsum(alt, 3, deq(s0.lo, s0.hi, 3), 2, deq(s3.lo, s3.hi, 3), 0, 0u);
                const3(k3, 1);
                sel3(t16, deq(f2.lo, f2.hi, 1), k3, alt);
                d3(t64, f3);
            } else {
                const int ui = -1, uj = t == 0 ? 0 : 1, vi = t == 0 ? -1 : 0, vj = 1;
                const Dig u2 = bdig(v, arr, 2, ui, uj), u3 = bdig(v, arr, 3, ui, uj), v2 = bdig(v, arr, 2, vi, vj),
                          v3 = bdig(v, arr, 3, vi, vj);
                cc = deq(u2.lo, u2.hi, 2);
                wsum(alt, 1, deq(u3.lo, u3.hi, 3), 3, deq(u2.lo, u2.hi, 3), 0, 0u);
                const3(k3, 2);
                sel3(t1, deq(f0.lo, f0.hi, 2), k3, alt);
                wsum(alt, 3, deq(v3.lo, v3.hi, 3), 2, deq(v2.lo, v2.hi, 3), 0, 0u);
                const3(k3, 1);
                sel3(t4, deq(f1.lo, f1.hi, 1), k3, alt);
                d3(t16, f2);
                d3(t64, f3);
            }
            uint32_t out[9];
            pack(out, t1, t4, t16, t64, cc);
#pragma unroll
            for (int k = 0; k < 9; ++k) v.st(arr, k, out[k], M);
            break;
        }
        case TD_BFLY_22: {
            const int p1 = (int)bb;
            const int want = t == 0 ? (p1 + 2) % 3 : (p1 + 1) % 3;
            const int arr = 5 + t;
            const uint32_t M = INT & slice3(t, i, c, want);
            const Dig f0 = bdig(v, arr, 0, 0, 0), f1 = bdig(v, arr, 1, 0, 0), f2 = bdig(v, arr, 2, 0, 0),
                      f3 = bdig(v, arr, 3, 0, 0);
            uint32_t t1[3], t4[3], t16[3], t64[3], cc, alt[3], k3[3];
            if (t == 2) {
                const Dig n1a = bdig(v, arr, 1, -1, 0), n1b = bdig(v, arr, 2, -1, 0);
                const uint32_t n2c = v.ld(arr, 8, 0, 1), n3c = v.ld(arr, 8, 1, 0);
                const Dig n4a = bdig(v, arr, 1, 0, -1), n4b = bdig(v, arr, 2, 0, -1);
                cc = deq(n1b.lo, n1b.hi, 1);
                wsum(alt, 3, deq(n1b.lo, n1b.hi, 3), 2, deq(n1a.lo, n1a.hi, 3), 0, 0u);
                const3(k3, 1);
                sel3(t1, deq(f0.lo, f0.hi, 1), k3, alt);
                d3(alt, f1.lo, f1.hi & f1.lo);  // (f1 != 2) * f1
                const3(k3, 2);
                sel3(t4, n2c, k3, alt);
                d3(alt, f2.lo & f2.hi, f2.hi);  // (f2 != 1) * f2
                const3(k3, 1);
                sel3(t16, n3c, k3, alt);
                wsum(alt, 1, deq(n4b.lo, n4b.hi, 3), 3, deq(n4a.lo, n4a.hi, 3), 0, 0u);
                const3(k3, 2);
                sel3(t64, deq(f3.lo, f3.hi, 2), k3, alt);
            } else {
                const int n1i = -1, n1j = t == 0 ? 0 : 1, n2i = t == 0 ? -1 : 0, n2j = 1;
                const int n3i = 1, n3j = t == 0 ? 0 : -1, n4i = t == 0 ? 1 : 0, n4j = -1;
                const uint32_t n1c = v.ld(arr, 8, n1i, n1j), n2c = v.ld(arr, 8, n2i, n2j);
                const Dig n30 = bdig(v, arr, 0, n3i, n3j), n31 = bdig(v, arr, 1, n3i, n3j);
                const Dig n40 = bdig(v, arr, 0, n4i, n4j), n41 = bdig(v, arr, 1, n4i, n4j);
                cc = deq(n30.lo, n30.hi, 2);
                d3(alt, f0.lo, f0.hi & f0.lo);  // (f0 != 2) * f0
                const3(k3, 2);
                sel3(t1, n1c, k3, alt);
                d3(alt, f1.lo & f1.hi, f1.hi);  // (f1 != 1) * f1
                const3(k3, 1);
                sel3(t4, n2c, k3, alt);
                wsum(alt, 3, deq(n30.lo, n30.hi, 3), 1, deq(n31.lo, n31.hi, 3), 0, 0u);
                const3(k3, 2);
                sel3(t16, deq(f2.lo, f2.hi, 2), k3, alt);
                wsum(alt, 2, deq(n40.lo, n40.hi, 3), 3, deq(n41.lo, n41.hi, 3), 0, 0u);
                const3(k3, 1);
                sel3(t64, deq(f3.lo, f3.hi, 1), k3, alt);
            }
            uint32_t out[9];
            pack(out, t1, t4, t16, t64, cc);
#pragma unroll
            for (int k = 0; k < 9; ++k) v.st(arr, k, out[k], M);
            break;
        }
        case TD_BFLY_23_LOZ: {
            const int p1 = (int)bb;
            const int want = t == 0 ? (p1 + 1) % 3 : (p1 + 2) % 3;
            const int arr = 5 + t;
            const uint32_t M = INT, S = INT & slice3(t, i, c, want);
            Dig d[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) d[k] = bdig(v, arr, k, 0, 0);
            const uint32_t cen = v.ld(arr, 8, 0, 0);
            Dig nd[4] = {d[0], d[1], d[2], d[3]};
            if (t == 2) {
                const uint32_t a = v.ld(arr, 8, -1, 0), b = v.ld(arr, 8, 0, -1);
                // t1 = a ? 1 : (f0 != 1) * f0; t64 = b ? 2 : (f3 != 2) * f3
                nd[0] = Dig{(a) | (d[0].lo & d[0].hi), ~a & d[0].hi};
                nd[3] = Dig{~b & d[3].lo, b | (d[3].hi & d[3].lo)};
            } else {
                const int n3i = 1, n3j = t == 0 ? 0 : -1, n4i = t == 0 ? 1 : 0, n4j = -1;
                const uint32_t a = v.ld(arr, 8, n3i, n3j), b = v.ld(arr, 8, n4i, n4j);
                // t16 = a ? 2 : (f2 != 2) * f2; t64 = b ? 1 : (f3 != 1) * f3
                nd[2] = Dig{~a & d[2].lo, a | (d[2].hi & d[2].lo)};
                nd[3] = Dig{b | (d[3].lo & d[3].hi), ~b & d[3].hi};
            }
            // the butterfly array after pass 23 (centre bit unchanged)
            Dig e[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) e[k] = Dig{(nd[k].lo & S) | (d[k].lo & ~S), (nd[k].hi & S) | (d[k].hi & ~S)};
            // UpdateLozengeFromButterflys{H,L,R} (:655-746), own site only
            const uint32_t o0 = deq(e[0].lo, e[0].hi, 3), o1 = deq(e[1].lo, e[1].hi, 3), o2 = deq(e[2].lo, e[2].hi, 3),
                           o3 = deq(e[3].lo, e[3].hi, 3);
            uint32_t H[4], L[4], R[4];
            if (t == 0) {
                H[0] = o0, H[1] = o1, H[2] = o2, H[3] = o3;
                L[0] = cen, L[1] = o2, L[2] = deq(e[3].lo, e[3].hi, 1), L[3] = deq(e[3].lo, e[3].hi, 2);
                R[0] = cen, R[1] = deq(e[2].lo, e[2].hi, 1), R[2] = deq(e[2].lo, e[2].hi, 2), R[3] = o3;
            } else if (t == 1) {
                L[0] = o0, L[1] = o1, L[2] = o2, L[3] = o3;
                R[0] = o0, R[1] = deq(e[1].lo, e[1].hi, 1), R[2] = deq(e[1].lo, e[1].hi, 2), R[3] = cen;
                H[0] = deq(e[0].lo, e[0].hi, 1), H[1] = deq(e[0].lo, e[0].hi, 2), H[2] = o1, H[3] = cen;
            } else {
                R[0] = o0, R[1] = o1, R[2] = o2, R[3] = o3;
                H[0] = deq(e[0].lo, e[0].hi, 1), H[1] = deq(e[0].lo, e[0].hi, 2), H[2] = cen, H[3] = o3;
                L[0] = o0, L[1] = cen, L[2] = deq(e[3].lo, e[3].hi, 1), L[3] = deq(e[3].lo, e[3].hi, 2);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v.st(arr, 2 * k, e[k].lo, S);
                v.st(arr, 2 * k + 1, e[k].hi, S);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v.st(0, k, H[k], M);
                v.st(1, k, L[k], M);
                v.st(2, k, R[k], M);
            }
            break;
        }
        default: break;
    }
}
}  // namespace tdp
}  // namespace rtb
