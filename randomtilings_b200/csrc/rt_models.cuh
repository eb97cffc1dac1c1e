// rt_models.cuh -- per-model site rules of the persistent walk kernel.
//
// A model maps a position (r, c) of the Rotate NDRange to its colour-array
// site and stream id, and applies one phase there:
//   OP_STEP  : if the previous phase flipped a different colour, first apply
//              that colour's pending Update at this site (the reference runs
//              Update right after every Rotate; when the same colour is
//              flipped twice in a row the first Update is overwritten by the
//              second before anything reads it, so it is skipped), then flip
//              the current colour with this position's draw;
//   OP_FINAL : apply the last colour's Update (end of the walk).
// Within one phase a site reads only the previously flipped colour at
// neighbouring sites (and its own old values), and writes the other colours
// at itself, so positions are independent and the result equals the
// reference's serial order.
//
// The rules read and write the CTA's shared-memory copy of the lattice
// through a Band view, indexed with the global (row, column) of the colour
// arrays.
#pragma once

#include "rt_device.cuh"

namespace rtb {

struct WalkArgs {
    void* arr[2][8];      // [lattice][colour] global colour arrays (2 lattices = coupled CFTP chains)
    int nlat;             // 1 or 2
    int n;                // tiling side N
    int rows, cols;       // Rotate NDRange (position grid)
    int arows, width;     // colour array shape
    int wpad;             // shared-memory row stride (elements, multiple of 4)
    int xwords;           // exchange words per row
    int xslots;           // exchanged arrays per phase (slots per side)
    int rows_per_cta;
    int rng_kind;         // 0 TinyMT, 1 Philox (fast mode)
    const uint4* params;  // TinyMT (mat1, mat2, tmat, -) per stream id, or nullptr
    uint32_t mat1, mat2, tmat;
    uint32_t chain;       // Philox counter word 3 (fast mode)
    const uint32_t* phases;
    int64_t nphases;
    const int64_t* epoch_start;  // first phase of each epoch
    const uint64_t* epoch_seed;  // per epoch: TinyMT seed (low 32 bits) or Philox key (fast mode)
    int nepochs;
    uint32_t thr[4];      // integer acceptance thresholds on the 23-bit draw
    float weights[16];    // rect-triangle face weights
    unsigned long long* xbuf;  // tagged halo-row exchange slots
    int* err;
    uint64_t timeout_ns;
    int64_t drop_phase;   // tests of the bounded waits: CTA 0 does not publish this phase's rows (-1: none)
    int depth;            // bit-plane kernel: phases per halo exchange
    int pwords;           // bit-plane kernel: 32-bit words per colour-array row
    int wper;             // periodic weights (domino heat bath, uniform lozenges): period P (1, 2, 4), 0 = none
    uint32_t wthr[16];    // ... the vertex's threshold at (i, j): wthr[(i mod P) P + (j mod P)]
};

// Threshold of a weighted rule at vertex (i, j): dominoes, the heat bath's
// draw below which the site becomes 12; lozenges, the draw below which a
// cube is added (removal stays below thr[1]).
__device__ __forceinline__ uint32_t weight_thr(const WalkArgs& a, int i, int j) {
    const int m = a.wper - 1;
    return a.wthr[(i & m) * a.wper + (j & m)];
}

// ---------------------------------------------------------------------------
// Model interface.  Per phase every thread builds a small context once (the
// decoded descriptor and the shared-memory planes it touches); per site the
// model gets the site's offset `off` inside a colour plane of the band, its
// global colour-array row i and column j, and the draw k.  Neighbours are
// off +- 1 (columns) and off +- w (rows); w = band row stride.
// ---------------------------------------------------------------------------

// Domino (src/Domino/DominoTiler.cpp:9-107; dominokernel.cl, dominokernelCFTP.cl).
// Colour 0 = black ((i+j) even), 1 = white, int8, N x N/2.  Position (r, c)
// of the (N-2) x (N/2-2) range is site (r+1, c+1), stream c + (N/2-2) r.
// Reference colour r flips array 1-r and then refreshes array r from it.
template <bool HEAT_BATH>
struct DominoRule {
    using Elem = int8_t;
    static constexpr int NCOL = 2;
    static constexpr int ROFF = 1;
    static constexpr int COFF = 1;
    // Array the reference's colour r flips (DominoTiler.cpp:36-41).
    __device__ static int flipped(int r) { return 1 - r; }
    __device__ static uint32_t stream_id(const WalkArgs& a, int r, int c) {
        return (uint32_t)c + (uint32_t)(a.n / 2 - 2) * (uint32_t)r;
    }
    struct Ctx {
        int8_t* dst;        // array written at the site
        const int8_t* src;  // flipped array whose neighbours are read
        int t;              // the reference's colour of the pending Update
        bool step, upd;
        int w;
        int arr;            // the array rotated (0 black, 1 white)
        uint32_t thr;
    };
    __device__ static uint32_t written(uint32_t d) { return ph_op(d) == OP_STEP ? 1u << flipped((int)ph_a(d)) : 0u; }
    __device__ static Ctx ctx(const WalkArgs& a, int8_t* planes, int plane, uint32_t d, int) {
        const int op = (int)ph_op(d), ca = (int)ph_a(d), cb = (int)ph_b(d);
        Ctx x;
        x.step = op == (int)OP_STEP;
        x.w = a.wpad;
        x.thr = a.thr[0];
        x.arr = 1 - ca;
        if (x.step) {
            x.upd = cb != (int)NO_COLOUR && cb != ca;
            x.dst = planes + (1 - ca) * plane;
            x.src = planes + ca * plane;
            x.t = cb;
        } else {
            x.upd = true;
            x.dst = planes + ca * plane;
            x.src = planes + (1 - ca) * plane;
            x.t = ca;
        }
        return x;
    }
    // Edge bits of a site from its four neighbours in the flipped array:
    // 1 up, 2 down, 4 towards j-1, 8 towards j+1 (dominokernel.cl:22-31).
    // The flipped array's neighbour towards j+1 shares the site's column in
    // rows of parity (i+t) odd, towards j-1 in the others.
    __device__ static int refreshed(const Ctx& x, int off, int i) {
        const int p = (i + x.t) & 1;
        const int up = x.src[off - x.w], down = x.src[off + x.w];
        const int west = x.src[off - (1 - p)], east = x.src[off + p];
        return ((up & 2) >> 1) | ((down & 1) << 1) | ((west & 8) >> 1) | ((east & 4) << 1);
    }
    // thr: draws below it act (ceil(0.8 * 2^23), or 2^22 for the heat bath).
    __device__ static int flip(int v, uint32_t k, uint32_t thr) {
        if (HEAT_BATH) return k < thr ? (v == 3 ? 12 : v) : (v == 12 ? 3 : v);
        return k < thr ? (v == 3 ? 12 : (v == 12 ? 3 : v)) : v;
    }
    __device__ static void site(const WalkArgs& a, const Ctx& x, int off, int i, int j, uint32_t k) {
        if (x.step) {
            const int v = x.upd ? refreshed(x, off, i) : (int)x.dst[off];
            // weighted heat bath: array column j is vertex column 2 j + ((i + arr) & 1)
            const uint32_t thr = HEAT_BATH && a.wper ? weight_thr(a, i, 2 * j + ((i + x.arr) & 1)) : x.thr;
            x.dst[off] = (int8_t)flip(v, k, thr);
        } else {
            x.dst[off] = (int8_t)refreshed(x, off, i);
        }
    }
};

// Shared skeleton of the three-colour models (lozenge, rect-triangle):
// arrays 0..2 of N x N/3, position (r, c) = site (r, c), stream c + (N/3) r;
// colour t's Update refreshes colours t+1 and t+2 (mod 3) at interior sites
// 1 <= i <= N-2, 1 <= j <= N/3-2.  `Rule::refresh` computes both refreshed
// values from the flipped array; the diagonal neighbours' column shifts
// depend on i mod 3 and are tabulated per phase (Rule::shift_table).
template <class T, class Rule>
struct ThreeColour {
    using Elem = T;
    static constexpr int NCOL = 3;
    static constexpr int ROFF = 0;
    static constexpr int COFF = 0;
    __device__ static int flipped(int r) { return r; }
    __device__ static uint32_t stream_id(const WalkArgs& a, int r, int c) {
        return (uint32_t)c + (uint32_t)(a.n / 3) * (uint32_t)r;
    }
    struct Ctx {
        T* cur;      // colour flipped in this phase (STEP)
        const T* f;  // colour whose Update is applied
        T* pa;       // colour t+1
        T* pb;       // colour t+2
        bool step, upd, keep_a;
        uint32_t shifts;
        int w, imax, jmax;
        int col;     // colour flipped (STEP)
    };
    __device__ static uint32_t written(uint32_t d) { return ph_op(d) == OP_STEP ? 1u << flipped((int)ph_a(d)) : 0u; }
    __device__ static Ctx ctx(const WalkArgs& a, T* planes, int plane, uint32_t d, int) {
        const int op = (int)ph_op(d), ca = (int)ph_a(d), cb = (int)ph_b(d);
        Ctx x;
        x.step = op == (int)OP_STEP;
        x.col = ca;
        x.w = a.wpad;
        x.imax = a.n - 2;
        x.jmax = a.n / 3 - 2;
        const int t = x.step ? cb : ca;
        x.upd = x.step ? (cb != (int)NO_COLOUR && cb != ca) : true;
        x.cur = planes + (x.step ? ca : 0) * plane;
        const int tt = x.upd ? t : 0;
        x.f = planes + tt * plane;
        x.pa = planes + ((tt + 1) % 3) * plane;
        x.pb = planes + ((tt + 2) % 3) * plane;
        x.keep_a = x.step && x.upd && (tt + 1) % 3 == ca;
        x.shifts = Rule::shift_table(tt);
        return x;
    }
    __device__ static void site(const WalkArgs& a, const Ctx& x, int off, int i, int j, uint32_t k) {
        const bool interior = i >= 1 && i <= x.imax && j >= 1 && j <= x.jmax;
        if (x.step) {
            int v;
            if (x.upd && interior) {
                int na, nb;
                Rule::refresh(x.f, off, x.w, (x.shifts >> (3 * (i % 3))) & 7u, (int)x.pa[off], (int)x.pb[off], na, nb);
                if (x.keep_a) {
                    v = na;
                    x.pb[off] = (T)nb;
                } else {
                    v = nb;
                    x.pa[off] = (T)na;
                }
            } else {
                v = (int)x.cur[off];
            }
            if constexpr (Rule::kSiteWeights) {
                // weighted lozenges: array column j of colour c is vertex column 3 j + (c + i) mod 3
                const uint32_t t0 = a.wper ? weight_thr(a, i, 3 * j + (x.col + i) % 3) : a.thr[0];
                x.cur[off] = (T)Rule::flip_w(v, k, t0, a.thr[1]);
            } else {
                x.cur[off] = (T)Rule::flip(v, k, a);
            }
        } else if (interior) {
            int na, nb;
            Rule::refresh(x.f, off, x.w, (x.shifts >> (3 * (i % 3))) & 7u, (int)x.pa[off], (int)x.pb[off], na, nb);
            x.pa[off] = (T)na;
            x.pb[off] = (T)nb;
        }
    }
};

// Lozenge (src/Lozenge/LozengeTiler.cpp:18-88; lozengekernel.cl, qlozengekernel.cl).
// Flippable vertices: 25 = 1+8+16 (no cube) and 38 = 2+4+32 (cube).
template <bool QWEIGHT>
struct LozengeRule {
    static constexpr bool kSiteWeights = !QWEIGHT;  // periodic weights on the uniform (char) kernel
    // UpdateTiles (lozengekernel.cl:36-54): colour t+1 refreshes bits {2,4,32},
    // colour t+2 bits {1,8,16}.  Per row class i mod 3: bit 0 = shift of the
    // upper-right / lower-left reads, bit 1 = of the left read, bit 2 = of
    // the right read.
    __device__ static uint32_t shift_table(int t) {
        uint32_t tab = 0;
        for (int rr = 0; rr < 3; ++rr) {
            const uint32_t sa = rr == (2 * t + 1) % 3, sw = rr == (2 * t + 2) % 3, se = rr == (2 * t) % 3;
            tab |= (sa | (sw << 1) | (se << 2)) << (3 * rr);
        }
        return tab;
    }
    template <class T>
    __device__ static void refresh(const T* f, int off, int w, uint32_t sh, int a_old, int b_old, int& na, int& nb) {
        const int sa = sh & 1, sw = (sh >> 1) & 1, se = (sh >> 2) & 1;
        na = (a_old & ~38) + (((int)f[off - w + sa] & 16) >> 3) + (((int)f[off - sw] & 8) >> 1) +
             (((int)f[off + w] & 1) << 5);
        nb = (b_old & ~25) + (((int)f[off - w] & 32) >> 5) + (((int)f[off + se] & 4) << 1) +
             (((int)f[off + w - sa] & 2) << 3);
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
    // The uniform rule with the add threshold of the site: k < t0 adds a
    // cube, t0 <= k < t1 removes one.
    __device__ static int flip_w(int v, uint32_t k, uint32_t t0, uint32_t t1) {
        if (k < t0) return v == 25 ? 38 : v;
        if (k < t1) return v == 38 ? 25 : v;
        return v;
    }
};

// Rectangle-triangle (src/RectTriangle/RectTriangleTiler.cpp:17-92;
// recttrianglekernel.cl).  A site holds six hex face digits.
struct RectTriRule {
    static constexpr bool kSiteWeights = false;
    __device__ static int digit(int x, int k) { return (int)(((unsigned)x >> (4 * k)) & 0xfu); }
    // updateTiles1 / updateTiles2 (recttrianglekernel.cl:120-146).  Per row
    // class: bit 0 = shift of the side read of colour t+1 (s1), bit 1 = of
    // the lower / upper-right reads (s2), bit 2 = of the side read of colour
    // t+2 (s3).
    __device__ static uint32_t shift_table(int t) {
        uint32_t tab = 0;
        for (int rr = 0; rr < 3; ++rr) {
            const uint32_t s1 = rr == t, s2 = rr == (t + 1) % 3, s3 = rr == (t + 2) % 3;
            tab |= (s1 | (s2 << 1) | (s3 << 2)) << (3 * rr);
        }
        return tab;
    }
    template <class T>
    __device__ static void refresh(const T* f, int off, int w, uint32_t sh, int, int, int& na, int& nb) {
        const int s1 = sh & 1, s2 = (sh >> 1) & 1, s3 = (sh >> 2) & 1;
        const int up = f[off - w], side = f[off + s1], low = f[off + w - s2];
        na = (digit(up, 1) << 20) | (digit(up, 0) << 16) | (digit(side, 5) << 12) | (digit(low, 4) << 8) |
             (digit(low, 3) << 4) | digit(side, 2);
        const int west = f[off - s3], upr = f[off - w + s2], down = f[off + w];
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
