// rt_models.cuh -- per-model site rules of the persistent walk kernel.
//
// A model maps a position (r, c) of the Rotate NDRange to its colour-array
// site, its TinyMT stream id, and applies one phase there:
//   OP_STEP  : if the previous phase flipped a different colour, first apply
//              that colour's pending Update at this site (the reference runs
//              Update right after every Rotate; when the same colour is
//              flipped twice in a row the first Update is overwritten by the
//              second before anything reads it, so it is skipped), then flip
//              the current colour with this position's draw;
//   OP_FINAL : apply the last colour's Update (end of the walk).
// Within one phase a site only reads the previously flipped colour at
// neighbouring sites and writes the other colours, so positions are
// independent and the kernel's result equals the reference's serial order.
#pragma once

#include "rt_device.cuh"

namespace rtb {

struct WalkArgs {
    void* arr[2][8];      // [lattice][colour] device arrays (2 lattices = coupled CFTP chains)
    int nlat;             // 1 or 2
    int n;                // tiling side N
    int rows, cols;       // Rotate NDRange (position grid)
    int rows_per_cta;
    int rng_kind;         // 0 TinyMT, 1 Philox
    const uint4* params;  // TinyMT (mat1, mat2, tmat, -) per stream id, or nullptr
    uint32_t mat1, mat2, tmat;
    uint32_t key0, key1;  // Philox key (fast mode)
    uint32_t chain;       // Philox counter word 3 (fast mode)
    const uint32_t* phases;
    int64_t nphases;
    const int64_t* epoch_start;  // first phase of each TinyMT epoch
    const uint32_t* epoch_seed;  // TinyMT seed of each epoch
    int nepochs;
    uint32_t thr[4];      // integer acceptance thresholds on the 23-bit draw
    float weights[16];    // rect-triangle face weights
    unsigned* flags;      // per-CTA count of completed phases
    int* err;
    uint64_t timeout_ns;
};

// ---------------------------------------------------------------------------
// Domino (src/Domino/DominoTiler.cpp:9-107; dominokernel.cl, dominokernelCFTP.cl).
// arr[0] = black ((i+j) even), arr[1] = white, int8, N x N/2.  Position
// (r, c) of the (N-2) x (N/2-2) range is site (r+1, c+1), stream c + (N/2-2) r.
// Reference colour r flips array 1-r and then refreshes array r from it.
// ---------------------------------------------------------------------------
template <bool HEAT_BATH>
struct DominoRule {
    __device__ static uint32_t stream_id(const WalkArgs& a, int r, int c) {
        return (uint32_t)c + (uint32_t)(a.n / 2 - 2) * (uint32_t)r;
    }
    // Edge bits of a site from its four neighbours in the flipped array:
    // 1 up, 2 down, 4 towards j-1, 8 towards j+1 (dominokernel.cl:22-31).
    __device__ static int refreshed(const int8_t* f, int i, int j, int h, int t) {
        const int up = ld_site(f + (i - 1) * h + j);
        const int down = ld_site(f + (i + 1) * h + j);
        const int west = ld_site(f + i * h + j - ((i + t + 1) & 1));
        const int east = ld_site(f + i * h + j + ((i + t) & 1));
        return ((up & 2) >> 1) | ((down & 1) << 1) | ((west & 8) >> 1) | ((east & 4) << 1);
    }
    // thr[0]: draws below it act (ceil(0.8 * 2^23), or 2^22 for the heat bath).
    __device__ static int flip(int v, uint32_t k, const WalkArgs& a) {
        if (HEAT_BATH) return k < a.thr[0] ? (v == 3 ? 12 : v) : (v == 12 ? 3 : v);
        return k < a.thr[0] ? (v == 3 ? 12 : (v == 12 ? 3 : v)) : v;
    }
    __device__ static void apply(const WalkArgs& a, uint32_t d, int r, int c, uint32_t k) {
        const int h = a.n / 2, i = r + 1, j = c + 1, at = i * h + j;
        const uint32_t op = ph_op(d), ca = ph_a(d), cb = ph_b(d);
        for (int l = 0; l < a.nlat; ++l) {
            if (op == OP_STEP) {
                int8_t* dst = static_cast<int8_t*>(a.arr[l][1 - ca]);
                const bool upd = cb != NO_COLOUR && cb != ca;
                const int v = upd ? refreshed(static_cast<const int8_t*>(a.arr[l][ca]), i, j, h, (int)cb)
                                  : ld_site(dst + at);
                const int nv = flip(v, k, a);
                if (upd || nv != v) st_site(dst + at, nv);
            } else {
                st_site(static_cast<int8_t*>(a.arr[l][ca]) + at,
                        refreshed(static_cast<const int8_t*>(a.arr[l][1 - ca]), i, j, h, (int)ca));
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Shared skeleton of the three-colour models (lozenge, rect-triangle):
// arrays arr[0..2] of N x N/3, position (r, c) = site (r, c), stream
// c + (N/3) r; colour t's Update refreshes colours t+1 and t+2 (mod 3) at
// interior sites 1 <= i <= N-2, 1 <= j <= N/3-2.
// ---------------------------------------------------------------------------
template <class T, class Rule>
struct ThreeColour {
    __device__ static uint32_t stream_id(const WalkArgs& a, int r, int c) {
        return (uint32_t)c + (uint32_t)(a.n / 3) * (uint32_t)r;
    }
    __device__ static void apply(const WalkArgs& a, uint32_t d, int r, int c, uint32_t k) {
        const int m = a.n / 3, i = r, j = c;
        const int at = i * m + j;
        const bool interior = i >= 1 && i <= a.n - 2 && j >= 1 && j <= m - 2;
        const uint32_t op = ph_op(d), ca = ph_a(d), cb = ph_b(d);
        for (int l = 0; l < a.nlat; ++l) {
            T* const* arr = reinterpret_cast<T* const*>(a.arr[l]);
            if (op == OP_STEP) {
                const bool upd = interior && cb != NO_COLOUR && cb != ca;
                int v;
                if (upd) {
                    const int ia = (int)(cb + 1) % 3, ib = (int)(cb + 2) % 3;
                    int na, nb;
                    Rule::refresh(arr[cb], i, j, m, (int)cb, ld_site(arr[ia] + at), ld_site(arr[ib] + at), na, nb, a);
                    if (ia == (int)ca) {
                        v = na;
                        st_site(arr[ib] + at, nb);
                    } else {
                        v = nb;
                        st_site(arr[ia] + at, na);
                    }
                } else {
                    v = ld_site(arr[ca] + at);
                }
                const int nv = Rule::flip(v, k, a);
                if (upd || nv != v) st_site(arr[ca] + at, nv);
            } else if (interior) {
                const int ia = (int)(ca + 1) % 3, ib = (int)(ca + 2) % 3;
                int na, nb;
                Rule::refresh(arr[ca], i, j, m, (int)ca, ld_site(arr[ia] + at), ld_site(arr[ib] + at), na, nb, a);
                st_site(arr[ia] + at, na);
                st_site(arr[ib] + at, nb);
            }
        }
    }
};

// Lozenge (src/Lozenge/LozengeTiler.cpp:18-88; lozengekernel.cl, qlozengekernel.cl).
// Flippable vertices: 25 = 1+8+16 (no cube) and 38 = 2+4+32 (cube).
template <class T, bool QWEIGHT>
struct LozengeRule {
    // UpdateTiles (lozengekernel.cl:36-54): colour t+1 refreshes bits {2,4,32},
    // colour t+2 bits {1,8,16}; the column shift of the diagonal neighbours
    // depends on i mod 3.
    template <class P>
    __device__ static void refresh(const P* f, int i, int j, int m, int t, int a_old, int b_old, int& na, int& nb,
                                   const WalkArgs&) {
        const int rr = i % 3;
        const int sa = rr == (2 * t + 1) % 3, sw = rr == (2 * t + 2) % 3, se = rr == (2 * t) % 3;
        na = (a_old & ~38) + ((ld_site(f + (i - 1) * m + j + sa) & 16) >> 3) + ((ld_site(f + i * m + j - sw) & 8) >> 1) +
             ((ld_site(f + (i + 1) * m + j) & 1) << 5);
        nb = (b_old & ~25) + ((ld_site(f + (i - 1) * m + j) & 32) >> 5) + ((ld_site(f + i * m + j + se) & 4) << 1) +
             ((ld_site(f + (i + 1) * m + j - sa) & 2) << 3);
    }
    // Uniform (lozengekernel.cl:3-34): thr[0] = ceil(.4 * 2^23) adds a cube,
    // thr[1] = ceil(.8 * 2^23) removes one.
    // q-weighted (qlozengekernel.cl:5-32): k < 2^22 proposes an add, accepted
    // iff k <= thr[0] = floor(q * 2^22); otherwise a removal, accepted iff
    // k - 2^22 <= thr[1] = floor((1/q) * 2^24), with q and 1/q in the
    // arithmetic (float32 or double) the comparison mode selects.
    __device__ static int flip(int v, uint32_t k, const WalkArgs& a) {
        if (!QWEIGHT) {
            if (k < a.thr[0]) return v == 25 ? 38 : v;
            if (k < a.thr[1]) return v == 38 ? 25 : v;
            return v;
        }
        if (k < (1u << 22)) return (v == 25 && k <= a.thr[0]) ? 38 : v;
        return (v == 38 && (k - (1u << 22)) <= a.thr[1]) ? 25 : v;
    }
};

// Rectangle-triangle (src/RectTriangle/RectTriangleTiler.cpp:17-92;
// recttrianglekernel.cl).  A site holds six hex face digits.
struct RectTriRule {
    __device__ static int digit(int x, int k) { return (int)(((unsigned)x >> (4 * k)) & 0xfu); }
    // updateTiles1 / updateTiles2 (recttrianglekernel.cl:120-146).
    template <class P>
    __device__ static void refresh(const P* f, int i, int j, int m, int t, int, int, int& na, int& nb, const WalkArgs&) {
        const int rr = i % 3;
        const int s1 = rr == t, s2 = rr == (t + 1) % 3, s3 = rr == (t + 2) % 3;
        const int up = ld_site(f + (i - 1) * m + j), side = ld_site(f + i * m + j + s1);
        const int low = ld_site(f + (i + 1) * m + j - s2);
        na = (digit(up, 1) << 20) | (digit(up, 0) << 16) | (digit(side, 5) << 12) | (digit(low, 4) << 8) |
             (digit(low, 3) << 4) | digit(side, 2);
        const int west = ld_site(f + i * m + j - s3), upr = ld_site(f + (i - 1) * m + j + s2);
        const int down = ld_site(f + (i + 1) * m + j);
        nb = (digit(west, 3) << 20) | (digit(upr, 2) << 16) | (digit(upr, 1) << 12) | (digit(west, 0) << 8) |
             (digit(down, 5) << 4) | digit(down, 4);
    }
    __device__ static float weight(const WalkArgs& a, int x) {
        float p = a.weights[digit(x, 5)];
        p = __fmul_rn(p, a.weights[digit(x, 4)]);
        p = __fmul_rn(p, a.weights[digit(x, 3)]);
        p = __fmul_rn(p, a.weights[digit(x, 2)]);
        p = __fmul_rn(p, a.weights[digit(x, 1)]);
        return __fmul_rn(p, a.weights[digit(x, 0)]);
    }
    // flipTiles (recttrianglekernel.cl:25-118): with probability 0.9f a site
    // proposes a move.  A member of the five-state hexagon cycle goes to the
    // state picked by the quarter of rd/0.9f (the member equal to itself
    // standing in for 0x122133); one of six pair states toggles to its
    // partner.  The move is kept iff weight(new)/weight(old) >= the draw
    // rescaled to [0,1).  IEEE float arithmetic, as on the host CPU.
    __device__ static int flip(int v, uint32_t k, const WalkArgs& a) {
        const float bs = 0.9f;
        float rd = __fsub_rn(__uint_as_float(k | 0x3f800000u), 1.0f);
        if (!(rd < bs)) return v;
        rd = __fdiv_rn(rd, bs);
        const int quarter = rd < 0.25f ? 0 : rd < 0.5f ? 1 : rd < 0.75f ? 2 : 3;
        float sc = (float)quarter * 0.25f;
        int nv = v;
        switch (v) {
            case 0x122133:
            case 0x331221:
            case 0x8ebbe8:
            case 0xfc99cf:
            case 0xa7dd7a: {
                const int pick = quarter == 0 ? 0xa7dd7a : quarter == 1 ? 0xfc99cf : quarter == 2 ? 0x8ebbe8 : 0x331221;
                nv = pick == v ? 0x122133 : pick;
                break;
            }
            case 0x47d47a: nv = 0xd22a33; sc = 1.0f; break;
            case 0xd22a33: nv = 0x47d47a; sc = 1.0f; break;
            case 0xa74d74: nv = 0x33a22d; sc = 1.0f; break;
            case 0x33a22d: nv = 0xa74d74; sc = 1.0f; break;
            case 0x8eb558: nv = 0x331eb1; sc = 1.0f; break;
            case 0x331eb1: nv = 0x8eb558; sc = 1.0f; break;
            case 0x855be8: nv = 0x1be133; sc = 1.0f; break;
            case 0x1be133: nv = 0x855be8; sc = 1.0f; break;
            case 0x6699cf: nv = 0xcf1221; sc = 1.0f; break;
            case 0xcf1221: nv = 0x6699cf; sc = 1.0f; break;
            case 0xfc9966: nv = 0x1221fc; sc = 1.0f; break;
            case 0x1221fc: nv = 0xfc9966; sc = 1.0f; break;
            default: return v;
        }
        const float ratio = __fdiv_rn(weight(a, nv), weight(a, v));
        const float x = sc == 1.0f ? rd : __fmul_rn(__fsub_rn(rd, sc), 4.0f);
        return ratio >= x ? nv : v;
    }
};

}  // namespace rtb
