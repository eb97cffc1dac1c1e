// rt_tridimer.cuh -- dimers on the triangular lattice (the reference's
// TriangleDimerTiler, src/TriangleDimer/TriangleDimerTiler.cpp:86-483 and
// triangledimerkernel.cl) as a phase program of the persistent walk kernel.
//
// Eight M x M int32 arrays (M = N/2), in band order:
//   0 H, 1 L, 2 R   lozenge states (one per edge orientation)
//   3 U, 4 D        up / down triangle states (three base-4 digits)
//   5 BH, 6 BL, 7 BR butterfly states (four base-4 digits + centre bit)
// The reference launches one kernel per array update; here each phase is
// one of those updates (or several that read only arrays finished in earlier
// phases and write different arrays), applied at every site, and a phase
// exchanges the halo rows of every array it wrote.  Position (i, j) of the
// (M, M) NDRange owns stream j + M i (src/TinyMT/tinymt.clh:24-30).
#pragma once

#include "rt_tdops.h"
#ifdef __CUDACC__
#include "rt_models.cuh"
#endif

namespace rtb {


struct TriDimerRule {
    using Elem = int32_t;
    static constexpr int NCOL = 8;
    static constexpr int ROFF = 0;
    static constexpr int COFF = 0;
    TD_HD static uint32_t stream_id(const WalkArgs& a, int r, int c) {
        return (uint32_t)c + (uint32_t)(a.n / 2) * (uint32_t)r;
    }
    // Arrays a phase writes (bit k = array k); their halo rows are exchanged.
    TD_HD static uint32_t written(uint32_t d) {
        const uint32_t op = ph_op(d), a = ph_a(d), b = ph_b(d);
        switch (op) {
            case TD_ROT_LOZ:
            case TD_LOZ_FLIPPED: return 1u << a;
            case TD_LOZ_OTHER: return 7u & ~(1u << a);
            case TD_UP_FROM_LOZ: return 1u << 3;
            case TD_TRI_OTHER: return (a == 0 ? 1u << 4 : 1u << 3) | (b << 5);
            case TD_ROT_TRI:
            case TD_TRI_FLIPPED: return a == 1 ? 1u << 4 : 1u << 3;
            case TD_LOZ_FROM_TRI: return 7u;
            case TD_BFLY_FROM_LOZ: return (b << 5) | (a ? 1u << 3 : 0u);
            case TD_ROT_BFLY:
            case TD_BFLY_SAME:
            case TD_BFLY_21:
            case TD_BFLY_22: return 1u << (5 + a);
            case TD_BFLY_23_LOZ: return (1u << (5 + a)) | 7u;
            default: return 0u;
        }
    }
    // Storage of the eight arrays: int32 planes of the walk kernels.  The
    // rule reads and writes values through get / set (accessors of other
    // layouts plug in the same way); the batch kernel keeps the arrays as
    // bit planes instead (rt_tdplane.cuh), with the same arithmetic.
    struct Ctx {
        int32_t* base;
        int plane, w, m, row0;
        uint32_t op, a, b;
        TD_HD int32_t get(int arr, int ii, int jj) const { return base[arr * plane + (ii - row0) * w + jj]; }
        TD_HD void set(int arr, int ii, int jj, int32_t v) const { base[arr * plane + (ii - row0) * w + jj] = v; }
    };
    TD_HD static Ctx ctx(const WalkArgs& ar, int32_t* planes, int plane, uint32_t d, int row0) {
        Ctx x;
        x.row0 = row0;
        x.base = planes;
        x.plane = plane;
        x.w = ar.wpad;
        x.m = ar.n / 2;
        x.op = ph_op(d);
        x.a = ph_a(d);
        x.b = ph_b(d);
        return x;
    }

    // ---- helpers ------------------------------------------------------------
    TD_HD static int dg(int32_t x, int k) { return (int)(((uint32_t)x >> (2 * k)) & 3u); }
    // 0->0, 1->2, 2->3, 3->1 and 0->0, 1->3, 2->1, 3->2 as 2-bit tables
    TD_HD static int cyc_up(int v) { return (int)((0x78u >> (2 * v)) & 3u); }
    TD_HD static int cyc_dn(int v) { return (int)((0x9Cu >> (2 * v)) & 3u); }
    TD_HD static int32_t pack(int t1, int t4, int t16, int t64, int c) {
        return t1 + 4 * t4 + 16 * t16 + 64 * t64 + 256 * c;
    }
    TD_HD static int tri_digit(int32_t v) {
        return ((v & 48) == 16 ? 1 : 0) + ((v & 3) == 3 ? 2 : 0) + ((v & 12) == 8 ? 3 : 0);
    }

    // Butterfly state of orientation `which` from the lozenge arrays
    // (UpdateButterflys{H,L,R}FromLozenge, triangledimerkernel.cl:118-189).
    template <class A>
    TD_HD static int32_t bfly_from_loz(const A& x, int which, int i, int j) {
        auto at = [&](int arr, int ii, int jj) { return x.get(arr, ii, jj); };
        int t1, t4, t16, t64, c;
        if (which == 0) {
            const int32_t h = at(0, i, j), ru = at(2, i - 1, j), lu = at(1, i - 1, j + 1), r = at(2, i, j), l = at(1, i, j);
            c = (lu >> 2) & 1;
            t1 = ((ru >> 3) & 1) + 2 * (ru & 1) + 3 * (h & 1);
            t4 = (lu & 1) + (lu & 2) + 3 * ((h >> 1) & 1);
            t16 = ((r >> 1) & 1) + ((r >> 1) & 2) + 3 * ((h >> 2) & 1);
            t64 = ((l >> 2) & 1) + ((l >> 2) & 2) + 3 * ((h >> 3) & 1);
        } else if (which == 1) {
            const int32_t l = at(1, i, j), h = at(0, i, j), r = at(2, i, j), hd = at(0, i + 1, j - 1), rw = at(2, i, j - 1);
            c = (r >> 3) & 1;
            t1 = (h & 1) + (h & 2) + 3 * (l & 1);
            t4 = ((r >> 1) & 1) + ((r >> 1) & 2) + 3 * ((l >> 1) & 1);
            t16 = ((hd >> 2) & 1) + ((hd >> 2) & 2) + 3 * ((l >> 2) & 1);
            t64 = ((rw >> 3) & 1) + 2 * (rw & 1) + 3 * ((l >> 3) & 1);
        } else {
            const int32_t r = at(2, i, j), h = at(0, i, j), le = at(1, i, j + 1), hd = at(0, i + 1, j), l = at(1, i, j);
            c = (le >> 3) & 1;
            t1 = (h & 1) + (h & 2) + 3 * (r & 1);
            t4 = (le & 1) + (le & 2) + 3 * ((r >> 1) & 1);
            t16 = ((hd >> 2) & 1) + ((hd >> 2) & 2) + 3 * ((r >> 2) & 1);
            t64 = ((l >> 2) & 1) + ((l >> 2) & 2) + 3 * ((r >> 3) & 1);
        }
        return pack(t1, t4, t16, t64, c);
    }

    // Up-triangle state from the lozenges (UpdateTriangleUFromLozenges, :96-116).
    template <class A>
    TD_HD static int32_t up_from_loz(const A& acc, int i, int j) {
        auto at = [&](int arr, int ii, int jj) { return acc.get(arr, ii, jj); };
        const int32_t l0 = at(1, i, j), l1 = at(1, i, j + 1), h0 = at(0, i, j), h1 = at(0, i + 1, j);
        const int x = ((l0 & 1) ? 1 : 0) + ((h0 & 8) ? 2 : 0) + ((h1 & 1) ? 3 : 0);
        const int y = ((l1 & 1) ? 1 : 0) + ((h1 & 2) ? 2 : 0) + ((l1 & 2) ? 3 : 0);
        const int z = ((l1 & 4) ? 1 : 0) + ((h1 & 8) ? 2 : 0) + ((h1 & 4) ? 3 : 0);
        return x + 4 * y + 16 * z;
    }

    TD_HD static int slice(int t, int i, int j) { return t == 0 ? i % 3 : t == 1 ? j % 3 : (i + j) % 3; }
    TD_HD static int bpar(int t, int i, int j) { return t == 1 ? (i & 1) : (j & 1); }

    TD_HD static void site(const WalkArgs&, const Ctx& x, int, int i, int j, uint32_t k) { site_on(x, i, j, k); }

    // One site of the phase whose op is OP (a compile-time constant: every
    // other case of the switch below folds away).  T >= 0 fixes the phase's
    // argument a (the orientation t) at compile time too, B >= 0 its
    // argument b; negative values read x.a / x.b.
    template <uint32_t OP, int T = -1, int B = -1, class A>
    TD_HD static void site_op(const A& x, int i, int j, uint32_t k) {
        auto at = [&](int arr, int ii, int jj) { return x.get(arr, ii, jj); };
        auto put = [&](int arr, int ii, int jj, int32_t v) { x.set(arr, ii, jj, v); };
        const bool interior = i >= 1 && i <= x.m - 2 && j >= 1 && j <= x.m - 2;
        const int t = T >= 0 ? T : (int)x.a;
        const uint32_t bm = B >= 0 ? (uint32_t)B : x.b;  // butterfly masks of TRI_OTHER / BFLY_FROM_LOZ
        switch (OP) {
            case TD_ROT_LOZ: {  // :4-22
                const int cls = ((1 - (t & 1)) * i + ((1 + t) / 2) * j) % 2;
                if (k < (1u << 22) && cls == (int)x.b) {
                    const int32_t v = at(t, i, j);
                    put(t, i, j, v == 5 ? 10 : v == 10 ? 5 : v);
                }
                break;
            }
            case TD_LOZ_FLIPPED: {  // :24-33
                const int cls = ((1 - (t & 1)) * i + ((1 + t) / 2) * j) % 2;
                if (!interior || cls == (int)x.b) break;
                const int dj = t & 1, di = (2 - t) / 2;
                put(t, i, j, ((at(t, i - 1, j + dj) >> 2) & 1) | (((at(t, i - di, j + 1) >> 3) & 1) << 1) |
                              ((at(t, i + 1, j - dj) & 1) << 2) | (((at(t, i + di, j - 1) >> 1) & 1) << 3));
                break;
            }
            case TD_LOZ_OTHER: {  // :35-78
                if (!interior) break;
                if (t == 0) {
                    put(1, i, j, (at(1, i, j) & ~10) | ((at(0, i + 1, j) & 1) << 1) | ((at(0, i + 1, j - 1) & 1) << 3));
                    put(2, i, j, (at(2, i, j) & ~10) | (at(0, i + 1, j) & 2) | (at(0, i, j) & 8));
                } else if (t == 1) {
                    put(2, i, j, (at(2, i, j) & ~5) | (at(1, i, j) & 1) | ((at(1, i + 1, j) & 1) << 2));
                    put(0, i, j, (at(0, i, j) & ~5) | ((at(1, i - 1, j) & 2) >> 1) | ((at(1, i, j) & 2) << 1));
                } else {
                    put(0, i, j, (at(0, i, j) & ~10) | (at(2, i - 1, j) & 2) | ((at(2, i, j - 1) & 2) << 2));
                    put(1, i, j, (at(1, i, j) & ~5) | (at(2, i, j) & 1) | (at(2, i, j - 1) & 4));
                }
                break;
            }
            case TD_UP_FROM_LOZ:
                if (interior) put(3, i, j, up_from_loz(x, i, j));
                break;
            case TD_TRI_OTHER: {  // :255-275, then :118-189 for the butterflies in b
                if (!interior) break;
                const int src = t == 0 ? 3 : 4, dst = t == 0 ? 4 : 3, p = t == 0 ? -1 : 1;
                // every value is computed before any is stored (the stores go to
                // arrays the computations do not read)
                const int32_t tv = tri_digit(at(src, i, j - 1 + t)) + 4 * tri_digit(at(src, i, j + t)) +
                                   16 * tri_digit(at(src, i + p, j));
                int32_t bv[3] = {0, 0, 0};
#pragma unroll
                for (int w = 0; w < 3; ++w)
                    if (bm & (1u << w)) bv[w] = bfly_from_loz(x, w, i, j);
                put(dst, i, j, tv);
#pragma unroll
                for (int w = 0; w < 3; ++w)
                    if (bm & (1u << w)) put(5 + w, i, j, bv[w]);
                break;
            }
            case TD_ROT_TRI: {  // :191-211
                if (k < (1u << 22) && (j + 2 * i) % 3 == (int)x.b) {
                    const int32_t v = at(t == 1 ? 4 : 3, i, j);
                    put(t == 1 ? 4 : 3, i, j, v == 45 ? 54 : v == 54 ? 45 : v);
                }
                break;
            }
            case TD_TRI_FLIPPED: {  // :213-253
                const int cls = (j + 2 * i) % 3;
                if (!interior || cls == (int)x.b) break;
                const int p = cls == ((int)x.b + 1) % 3;
                const int arr = t == 1 ? 4 : 3;
                int32_t v;
                if (t == 0)
                    v = p ? dg(at(arr, i, j - 1), 1) + 4 * dg(at(arr, i - 1, j + 1), 2) + 16 * dg(at(arr, i + 1, j), 0)
                          : dg(at(arr, i - 1, j), 2) + 4 * dg(at(arr, i, j + 1), 0) + 16 * dg(at(arr, i + 1, j - 1), 1);
                else
                    v = p ? dg(at(arr, i, j - 1), 1) + 4 * dg(at(arr, i + 1, j), 2) + 16 * dg(at(arr, i - 1, j + 1), 0)
                          : dg(at(arr, i + 1, j - 1), 2) + 4 * dg(at(arr, i, j + 1), 0) + 16 * dg(at(arr, i - 1, j), 1);
                put(arr, i, j, v);
                break;
            }
            case TD_LOZ_FROM_TRI: {  // :277-329
                if (!interior) break;
                const int32_t dd = at(4, i, j), uh = at(3, i - 1, j), ul = at(3, i, j - 1), ur = at(3, i, j);
                put(0, i, j, ((dd & 48) == 32) + 2 * ((dd & 48) == 48) + 4 * ((uh & 48) == 48) + 8 * ((uh & 48) == 32));
                put(1, i, j, ((ul & 12) == 4) + 2 * ((ul & 12) == 12) + 4 * ((dd & 3) == 1) + 8 * ((dd & 3) == 2));
                put(2, i, j, ((ur & 3) == 1) + 2 * ((dd & 12) == 12) + 4 * ((dd & 12) == 4) + 8 * ((ur & 3) == 2));
                break;
            }
            case TD_BFLY_FROM_LOZ: {
                if (!interior) break;
                int32_t bv[3] = {0, 0, 0};
#pragma unroll
                for (int w = 0; w < 3; ++w)
                    if (bm & (1u << w)) bv[w] = bfly_from_loz(x, w, i, j);
                const int32_t uv = t ? up_from_loz(x, i, j) : 0;  // a = 1: also U from the lozenges
#pragma unroll
                for (int w = 0; w < 3; ++w)
                    if (bm & (1u << w)) put(5 + w, i, j, bv[w]);
                if (t) put(3, i, j, uv);
                break;
            }
            case TD_ROT_BFLY: {  // :331-353
                const int p1 = (int)(x.b & 3), p2 = (int)(x.b >> 2);
                const int b1 = 1 - (t & 1), b2 = (1 + t) / 2, b3 = t & 1;
                if (k < (1u << 22) && (b1 * i + b2 * j) % 3 == p1 && ((b1 * j + b3 * i) & 1) == p2) {
                    const int32_t v = at(5 + t, i, j);
                    put(5 + t, i, j, v == 170 ? 85 : v == 85 ? 170 : v);
                }
                break;
            }
            case TD_BFLY_SAME: {  // UpdateButterflysFlipped{H,L,R}1
                const int p1 = (int)(x.b & 3), p2 = (int)(x.b >> 2);
                if (!interior || slice(t, i, j) != p1 || bpar(t, i, j) == p2) break;
                const int arr = 5 + t;
                const int c = (at(arr, i, j) >> 8) & 1;
                int t1, t4, t16, t64;
                if (t == 2) {
                    const int32_t lo = at(arr, i + 1, j - 1), hi = at(arr, i - 1, j + 1);
                    t1 = cyc_dn(dg(hi, 3));
                    t4 = cyc_up(dg(hi, 2));
                    t16 = cyc_dn(dg(lo, 1));
                    t64 = cyc_up(dg(lo, 0));
                } else {
                    const int32_t u = t == 0 ? at(arr, i, j - 1) : at(arr, i - 1, j);
                    const int32_t v = t == 0 ? at(arr, i, j + 1) : at(arr, i + 1, j);
                    t1 = cyc_up(dg(u, 1));
                    t4 = cyc_dn(dg(v, 0));
                    t16 = cyc_up(dg(v, 3));
                    t64 = cyc_dn(dg(u, 2));
                }
                put(arr, i, j, pack(t1, t4, t16, t64, c));
                break;
            }
            case TD_BFLY_21: {
                const int p1 = (int)x.b;
                const int want = t == 0 ? (p1 + 1) % 3 : (p1 + 2) % 3;
                if (!interior || slice(t, i, j) != want) break;
                const int arr = 5 + t;
                const int32_t f = at(arr, i, j);
                int t1, t4, t16, t64, c;
                if (t == 2) {
                    const int32_t e = at(arr, i, j + 1), s = at(arr, i + 1, j);
                    c = dg(s, 0) == 1;
                    t1 = dg(f, 0);
                    t4 = dg(f, 1) == 2 ? 2 : (dg(e, 0) == 3) + 3 * (dg(e, 3) == 3);
                    t16 = dg(f, 2) == 1 ? 1 : 3 * (dg(s, 0) == 3) + 2 * (dg(s, 3) == 3);
                    t64 = dg(f, 3);
                } else {
                    const int32_t u = t == 0 ? at(arr, i - 1, j) : at(arr, i - 1, j + 1);
                    const int32_t v = t == 0 ? at(arr, i - 1, j + 1) : at(arr, i, j + 1);
                    c = dg(u, 2) == 2;
                    t1 = dg(f, 0) == 2 ? 2 : (dg(u, 3) == 3) + 3 * (dg(u, 2) == 3);
                    t4 = dg(f, 1) == 1 ? 1 : 3 * (dg(v, 3) == 3) + 2 * (dg(v, 2) == 3);
                    t16 = dg(f, 2);
                    t64 = dg(f, 3);
                }
                put(arr, i, j, pack(t1, t4, t16, t64, c));
                break;
            }
            case TD_BFLY_22: {
                const int p1 = (int)x.b;
                const int want = t == 0 ? (p1 + 2) % 3 : (p1 + 1) % 3;
                if (!interior || slice(t, i, j) != want) break;
                const int arr = 5 + t;
                const int32_t f = at(arr, i, j);
                int t1, t4, t16, t64, c;
                if (t == 2) {
                    const int32_t n1 = at(arr, i - 1, j), n2 = at(arr, i, j + 1), n3 = at(arr, i + 1, j), n4 = at(arr, i, j - 1);
                    c = dg(n1, 2) == 1;
                    t1 = dg(f, 0) == 1 ? 1 : 3 * (dg(n1, 2) == 3) + 2 * (dg(n1, 1) == 3);
                    t4 = (n2 & 256) ? 2 : (dg(f, 1) != 2) * dg(f, 1);
                    t16 = (n3 & 256) ? 1 : (dg(f, 2) != 1) * dg(f, 2);
                    t64 = dg(f, 3) == 2 ? 2 : (dg(n4, 2) == 3) + 3 * (dg(n4, 1) == 3);
                } else {
                    const int32_t n1 = t == 0 ? at(arr, i - 1, j) : at(arr, i - 1, j + 1);
                    const int32_t n2 = t == 0 ? at(arr, i - 1, j + 1) : at(arr, i, j + 1);
                    const int32_t n3 = t == 0 ? at(arr, i + 1, j) : at(arr, i + 1, j - 1);
                    const int32_t n4 = t == 0 ? at(arr, i + 1, j - 1) : at(arr, i, j - 1);
                    c = dg(n3, 0) == 2;
                    t1 = (n1 & 256) ? 2 : (dg(f, 0) != 2) * dg(f, 0);
                    t4 = (n2 & 256) ? 1 : (dg(f, 1) != 1) * dg(f, 1);
                    t16 = dg(f, 2) == 2 ? 2 : 3 * (dg(n3, 0) == 3) + (dg(n3, 1) == 3);
                    t64 = dg(f, 3) == 1 ? 1 : 2 * (dg(n4, 0) == 3) + 3 * (dg(n4, 1) == 3);
                }
                put(arr, i, j, pack(t1, t4, t16, t64, c));
                break;
            }
            case TD_BFLY_23_LOZ: {
                if (!interior) break;
                const int p1 = (int)x.b;
                const int want = t == 0 ? (p1 + 1) % 3 : (p1 + 2) % 3;
                const int arr = 5 + t;
                if (slice(t, i, j) == want) {
                    const int32_t f = at(arr, i, j);
                    int t1 = dg(f, 0), t4 = dg(f, 1), t16 = dg(f, 2), t64 = dg(f, 3);
                    if (t == 2) {
                        t1 = (at(arr, i - 1, j) & 256) ? 1 : (dg(f, 0) != 1) * dg(f, 0);
                        t64 = (at(arr, i, j - 1) & 256) ? 2 : (dg(f, 3) != 2) * dg(f, 3);
                    } else {
                        const int32_t n3 = t == 0 ? at(arr, i + 1, j) : at(arr, i + 1, j - 1);
                        const int32_t n4 = t == 0 ? at(arr, i + 1, j - 1) : at(arr, i, j - 1);
                        t16 = (n3 & 256) ? 2 : (dg(f, 2) != 2) * dg(f, 2);
                        t64 = (n4 & 256) ? 1 : (dg(f, 3) != 1) * dg(f, 3);
                    }
                    put(arr, i, j, pack(t1, t4, t16, t64, (f >> 8) & 1));
                }
                // UpdateLozengeFromButterflys{H,L,R} (:655-746), own site only.
                const int32_t bf = at(arr, i, j);
                const int d0 = dg(bf, 0), d1 = dg(bf, 1), d2 = dg(bf, 2), d3 = dg(bf, 3), c = (bf >> 8) & 1;
                const int32_t own = (d0 == 3) + 2 * (d1 == 3) + 4 * (d2 == 3) + 8 * (d3 == 3);
                if (t == 0) {
                    put(0, i, j, own);
                    put(1, i, j, c + 2 * (d2 == 3) + 4 * (d3 == 1) + 8 * (d3 == 2));
                    put(2, i, j, c + 2 * (d2 == 1) + 4 * (d2 == 2) + 8 * (d3 == 3));
                } else if (t == 1) {
                    put(1, i, j, own);
                    put(2, i, j, (d0 == 3) + 2 * (d1 == 1) + 4 * (d1 == 2) + 8 * c);
                    put(0, i, j, (d0 == 1) + 2 * (d0 == 2) + 4 * (d1 == 3) + 8 * c);
                } else {
                    put(2, i, j, own);
                    put(0, i, j, (d0 == 1) + 2 * (d0 == 2) + 4 * c + 8 * (d3 == 3));
                    put(1, i, j, (d0 == 3) + 2 * c + 4 * (d3 == 1) + 8 * (d3 == 2));
                }
                break;
            }
            default: break;
        }
    }

    template <class A>
    TD_HD static void site_on(const A& x, int i, int j, uint32_t k) {
        switch (x.op) {
            case TD_ROT_LOZ: site_op<TD_ROT_LOZ>(x, i, j, k); break;
            case TD_LOZ_FLIPPED: site_op<TD_LOZ_FLIPPED>(x, i, j, k); break;
            case TD_LOZ_OTHER: site_op<TD_LOZ_OTHER>(x, i, j, k); break;
            case TD_UP_FROM_LOZ: site_op<TD_UP_FROM_LOZ>(x, i, j, k); break;
            case TD_TRI_OTHER: site_op<TD_TRI_OTHER>(x, i, j, k); break;
            case TD_ROT_TRI: site_op<TD_ROT_TRI>(x, i, j, k); break;
            case TD_TRI_FLIPPED: site_op<TD_TRI_FLIPPED>(x, i, j, k); break;
            case TD_LOZ_FROM_TRI: site_op<TD_LOZ_FROM_TRI>(x, i, j, k); break;
            case TD_BFLY_FROM_LOZ: site_op<TD_BFLY_FROM_LOZ>(x, i, j, k); break;
            case TD_ROT_BFLY: site_op<TD_ROT_BFLY>(x, i, j, k); break;
            case TD_BFLY_SAME: site_op<TD_BFLY_SAME>(x, i, j, k); break;
            case TD_BFLY_21: site_op<TD_BFLY_21>(x, i, j, k); break;
            case TD_BFLY_22: site_op<TD_BFLY_22>(x, i, j, k); break;
            case TD_BFLY_23_LOZ: site_op<TD_BFLY_23_LOZ>(x, i, j, k); break;
            default: break;
        }
    }

    // The rows of phase (OP, a, b) that can hold a changing site: those with
    // i = o (mod S).  Phases whose class condition depends on the row alone
    // (i mod 2 or i mod 3 for orientation 0, i mod 2 for some of
    // orientation 1) skip the other rows; all others have S = 1.
    template <uint32_t OP>
    TD_HD static void live_rows(uint32_t a, uint32_t b, int* S, int* o) {
        const int t = (int)a;
        *S = 1;
        *o = 0;
        if (OP == TD_ROT_LOZ && t == 0) *S = 2, *o = (int)b;             // class i mod 2 == b
        if (OP == TD_LOZ_FLIPPED && t == 0) *S = 2, *o = 1 - (int)b;     // class i mod 2 != b
        if (OP == TD_ROT_BFLY || OP == TD_BFLY_SAME) {
            const int p1 = (int)(b & 3), p2 = (int)(b >> 2);
            if (t == 0) *S = 3, *o = p1;                                    // slice i mod 3 == p1
            if (t == 1) *S = 2, *o = OP == TD_ROT_BFLY ? p2 : 1 - p2;      // parity i mod 2
        }
        if (OP == TD_BFLY_21 && t == 0) *S = 3, *o = ((int)b + 1) % 3;
        if (OP == TD_BFLY_22 && t == 0) *S = 3, *o = ((int)b + 2) % 3;
    }
};

}  // namespace rtb
