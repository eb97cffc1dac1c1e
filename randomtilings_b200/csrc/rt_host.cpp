// rt_host.cpp -- host-side domains, extremal tilings and height functions.
//
// These are the static helpers of the reference's Tiler classes, rewritten as
// plain C++ behind the C ABI.  Domain / tiling encodings and the height
// normalisation (h = 0 at the first boundary vertex in row-major order,
// INT_MAX outside the domain) are the reference's, so results are
// interchangeable with it.  Extremal tilings follow Thurston's construction:
// boundary heights by a walk along the boundary, then the extremal height
// function as a shortest-path flood that only moves in the height-increasing
// (max) or -decreasing (min) direction, then the tiling from height
// differences.  A domain that is not tileable is reported (RT_E_INVAL); the
// reference prints a message and returns a partial result instead.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <deque>
#include <map>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/rt_b200.h"
#include "../../include/rt_b200_host.h"
#include "rt_guard.h"

using rtb::guarded;

namespace {

constexpr int32_t INF = INT_MAX;
using Vec = std::vector<int32_t>;

// The largest side of a square array any function here takes or builds:
// 2 kMaxSide^2 (a lozenge domain's entries) still fits an int32 index.
constexpr int64_t kMaxSide = 32767;

// The side of a square array of n entries; -1 if n is not a square or the
// side exceeds kMaxSide.
int isqrt_exact(int64_t n) {
    if (n < 0 || n > (int64_t)1 << 40) return -1;
    int64_t r = (int64_t)std::llround(std::sqrt((double)n));
    while (r * r > n) --r;
    while ((r + 1) * (r + 1) <= n) ++r;
    return r * r == n && r <= kMaxSide ? (int)r : -1;
}

rt_status emit(const Vec& v, int32_t* out, int64_t cap, int64_t* len) {
    if (len) *len = (int64_t)v.size();
    if (!out) return RT_OK;
    if (cap < (int64_t)v.size()) return RT_E_INVAL;
    std::copy(v.begin(), v.end(), out);
    return RT_OK;
}

// Size queries (out == NULL) of the functions whose length follows from the
// input sizes: nothing else is computed.
rt_status size_only(int64_t n, int64_t* len) {
    if (len) *len = n;
    return RT_OK;
}
// Extremal tilings: the (M+1) x (M+1) vertices of an M x M domino domain ...
rt_status dom_side_query(int64_t dlen, int64_t* len) {
    const int m = isqrt_exact(dlen);
    return m < 1 ? RT_E_INVAL : size_only((int64_t)(m + 1) * (m + 1), len);
}
// ... or of an M x 2M lozenge domain.
rt_status loz_side_query(int64_t dlen, int64_t* len) {
    const int m = isqrt_exact(dlen / 2);
    return (m < 2 || (int64_t)2 * m * m != dlen) ? RT_E_INVAL : size_only((int64_t)(m + 1) * (m + 1), len);
}

// Dijkstra with unit steps from all seeded vertices; `dir` = +1 grows heights
// from the lowest (maximal height function), -1 shrinks them from the highest
// (minimal one).  allowed(v, nb) says whether the move v -> nb is one that
// changes the height by `dir`.
template <class Neighbours, class Allowed>
bool extremal_flood(Vec& hf, const Vec& verts, const std::vector<int>& seeds, int dir, Neighbours nbrs,
                    Allowed allowed) {
    std::map<int64_t, std::vector<int>> buckets;  // height -> vertices (processed lowest first for dir > 0)
    for (int v : seeds) buckets[(int64_t)dir * hf[v]].push_back(v);
    while (!buckets.empty()) {
        auto it = buckets.begin();
        std::vector<int> level;
        level.swap(it->second);
        buckets.erase(it);
        for (size_t k = 0; k < level.size(); ++k) {
            const int v = level[k];
            int nb[8], cnt = nbrs(v, nb);
            for (int e = 0; e < cnt; ++e) {
                const int w = nb[e];
                if (w < 0 || verts[w] == 0 || !allowed(v, e)) continue;
                const int32_t h = hf[v] + dir;
                if (verts[w] == 2) {
                    // A boundary height may not exceed (max) / undercut (min) the flood.
                    if (verts[v] != 2 && (int64_t)dir * hf[w] > (int64_t)dir * h) return false;
                } else if (hf[w] == INF) {
                    hf[w] = h;
                    buckets[(int64_t)dir * h].push_back(w);
                }
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Dominoes (src/Domino/DominoTiler.cpp).  Domain: M x M faces; tiling and
// heights on the (M+1) x (M+1) vertices; vertex bits 1 up, 2 down, 8 towards
// j+1, 4 towards j-1.
// ---------------------------------------------------------------------------
const int kDomDi[4] = {1, -1, 0, 0};
const int kDomDj[4] = {0, 0, 1, -1};
const int kDomBit[4] = {2, 1, 8, 4};

int dom_face(const Vec& d, int m, int i, int j) { return (i >= 0 && j >= 0 && i < m && j < m) ? d[i * m + j] : 0; }

// The two faces on either side of the edge from vertex (i, j) in direction nb.
void dom_edge_faces(int i, int j, int nb, int f[4]) {
    switch (nb) {
        case 0: f[0] = i, f[1] = j - 1, f[2] = i, f[3] = j; break;
        case 1: f[0] = i - 1, f[1] = j - 1, f[2] = i - 1, f[3] = j; break;
        case 2: f[0] = i - 1, f[1] = j, f[2] = i, f[3] = j; break;
        default: f[0] = i - 1, f[1] = j - 1, f[2] = i, f[3] = j - 1; break;
    }
}

// Height change along an edge, checkerboard rule of DominoTiler.cpp:221-231.
int dom_dh(int i, int j, int nb) { return (nb > 1 ? 1 : -1) * (((i + j) % 2 == 0) ? 1 : -1); }

int dom_face_p(const int32_t* d, int m, int i, int j) {
    return (i >= 0 && j >= 0 && i < m && j < m) ? d[(int64_t)i * m + j] : 0;
}

// Kind of vertex (i, j): 0 outside the domain, 1 interior (all four faces in
// it), 2 boundary (DomainToVertices, DominoTiler.cpp:479-506).
int dom_vertex_kind(const int32_t* d, int m, int i, int j) {
    if (i == 0 || j == 0 || i == m || j == m) {
        const int i0 = i - (i == m), i1 = i - 1 + (i == 0), j0 = j - (j == m), j1 = j - 1 + (j == 0);
        return (dom_face_p(d, m, i0, j0) || dom_face_p(d, m, i1, j0) || dom_face_p(d, m, i0, j1) ||
                dom_face_p(d, m, i1, j1))
                   ? 2
                   : 0;
    }
    const int s = (d[(int64_t)(i - 1) * m + j - 1] != 0) + (d[(int64_t)(i - 1) * m + j] != 0) +
                  (d[(int64_t)i * m + j - 1] != 0) + (d[(int64_t)i * m + j] != 0);
    return s == 4 ? 1 : s > 0 ? 2 : 0;
}

Vec dom_vertices(const Vec& d, int m) {
    const int n = m + 1;
    Vec v((size_t)n * n, 0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) v[(size_t)i * n + j] = dom_vertex_kind(d.data(), m, i, j);
    return v;
}

int first_boundary(const Vec& verts) {
    for (size_t k = 0; k < verts.size(); ++k)
        if (verts[k] == 2) return (int)k;
    return -1;
}

Vec dom_height_to_tiling(const Vec& hf, const Vec& d, int n) {
    const int m = n - 1;
    Vec t((size_t)n * n, 0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            if (hf[i * n + j] == INF) continue;
            for (int nb = 0; nb < 4; ++nb) {
                const int i2 = i + kDomDi[nb], j2 = j + kDomDj[nb];
                if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n || hf[i2 * n + j2] == INF) continue;
                int f[4];
                dom_edge_faces(i, j, nb, f);
                if (!dom_face(d, m, f[0], f[1]) && !dom_face(d, m, f[2], f[3])) continue;
                const int64_t diff = (int64_t)hf[i2 * n + j2] - hf[i * n + j];
                // modulo 2^32, so that heights that are no height function
                // (any int32 input) still give a defined result
                int32_t& tv = t[(size_t)i * n + j];
                tv = (int32_t)((uint32_t)tv + (uint32_t)kDomBit[nb] * (uint32_t)std::llabs(diff / 2));
            }
        }
    return t;
}

rt_status dom_extremal(const Vec& d, int dir, Vec* out) {
    const int m = isqrt_exact((int64_t)d.size());
    if (m < 1) return RT_E_INVAL;
    const int n = m + 1;
    const Vec verts = dom_vertices(d, m);
    Vec hf((size_t)n * n, INF);
    const int start = first_boundary(verts);
    if (start < 0) return RT_E_INVAL;
    hf[start] = 0;
    // Boundary heights: walk along boundary edges (exactly one adjacent face in the domain).
    std::deque<int> q{start};
    std::vector<int> seeds{start};
    while (!q.empty()) {
        const int v = q.front();
        q.pop_front();
        const int i = v / n, j = v % n;
        for (int nb = 0; nb < 4; ++nb) {
            const int i2 = i + kDomDi[nb], j2 = j + kDomDj[nb];
            if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n || verts[i2 * n + j2] != 2) continue;
            int f[4];
            dom_edge_faces(i, j, nb, f);
            if ((dom_face(d, m, f[0], f[1]) != 0) == (dom_face(d, m, f[2], f[3]) != 0)) continue;
            const int w = i2 * n + j2;
            const int32_t h = hf[v] + dom_dh(i, j, nb);
            if (hf[w] == INF) {
                hf[w] = h;
                q.push_back(w);
                seeds.push_back(w);
            } else if (hf[w] != h) {
                return RT_E_INVAL;  // boundary heights inconsistent: not tileable
            }
        }
    }
    auto nbrs = [&](int v, int* out4) {
        const int i = v / n, j = v % n;
        for (int nb = 0; nb < 4; ++nb) {
            const int i2 = i + kDomDi[nb], j2 = j + kDomDj[nb];
            out4[nb] = (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n) ? -1 : i2 * n + j2;
        }
        return 4;
    };
    auto allowed = [&](int v, int nb) { return dom_dh(v / n, v % n, nb) == dir; };
    if (!extremal_flood(hf, verts, seeds, dir, nbrs, allowed)) return RT_E_INVAL;
    *out = dom_height_to_tiling(hf, d, n);
    return RT_OK;
}

// ---------------------------------------------------------------------------
// Lozenges (src/Lozenge/LozengeTiler.cpp).  Domain: M rows of 2M triangles;
// tiling and heights on the (M+1) x (M+1) vertices of the triangular
// lattice; six neighbours with height steps -1, +1, ... and bits 8, 2, 1, 4,
// 16, 32 (LozengeTiler.cpp:12-16).
// ---------------------------------------------------------------------------
const int kLozDi[6] = {0, -1, -1, 0, 1, 1};
const int kLozDj[6] = {1, 1, 0, -1, -1, 0};
const int kLozDh[6] = {-1, 1, -1, 1, -1, 1};
const int kLozBit[6] = {8, 2, 1, 4, 16, 32};
// (row offset, offset from 2j) of the two triangles beside edge nb.
const int kLozFace[6][4] = {{0, 0, -1, 1}, {-1, 1, -1, 0}, {-1, 0, -1, -1}, {-1, -1, 0, -2}, {0, -2, 0, -1}, {0, -1, 0, 0}};

int loz_face_p(const int32_t* d, int m, int r, int c) {
    return (r >= 0 && c >= 0 && r < m && c < 2 * m) ? d[(int64_t)r * 2 * m + c] : 0;
}
int loz_face(const Vec& d, int m, int r, int c) { return loz_face_p(d.data(), m, r, c); }

bool loz_edge_in_p(const int32_t* d, int m, int i, int j, int nb, bool exclusive) {
    const int a = loz_face_p(d, m, i + kLozFace[nb][0], 2 * j + kLozFace[nb][1]) != 0;
    const int b = loz_face_p(d, m, i + kLozFace[nb][2], 2 * j + kLozFace[nb][3]) != 0;
    return exclusive ? (a != b) : (a || b);
}
bool loz_edge_in(const Vec& d, int m, int i, int j, int nb, bool exclusive) {
    return loz_edge_in_p(d.data(), m, i, j, nb, exclusive);
}

// Kind of vertex (i, j) from its six triangles (DomainToVertices,
// LozengeTiler.cpp:405-430); the border rows and columns are outside.
int loz_vertex_kind(const int32_t* d, int m, int i, int j) {
    if (i < 1 || j < 1 || i >= m || j >= m) return 0;
    const int64_t r = (int64_t)i * 2 * m, u = (int64_t)(i - 1) * 2 * m;
    const int s = (d[r + 2 * j] != 0) + (d[r + 2 * j - 1] != 0) + (d[r + 2 * j - 2] != 0) + (d[u + 2 * j] != 0) +
                  (d[u + 2 * j + 1] != 0) + (d[u + 2 * j - 1] != 0);
    return s == 6 ? 1 : s > 0 ? 2 : 0;
}

Vec loz_vertices(const Vec& d, int m) {
    const int n = m + 1;
    Vec v((size_t)n * n, 0);
    for (int i = 1; i < m; ++i)
        for (int j = 1; j < m; ++j) v[(size_t)i * n + j] = loz_vertex_kind(d.data(), m, i, j);
    return v;
}

Vec loz_height_to_tiling(const Vec& hf, const Vec& d, int n) {
    const int m = n - 1;
    Vec t((size_t)n * n, 0);
    for (int i = 1; i < n - 1; ++i)
        for (int j = 1; j < n - 1; ++j)
            for (int nb = 0; nb < 6; ++nb) {
                if (!loz_edge_in(d, m, i, j, nb, false)) continue;
                const int i2 = i + kLozDi[nb], j2 = j + kLozDj[nb];
                if (std::llabs((int64_t)hf[i2 * n + j2] - hf[i * n + j]) == 2) t[i * n + j] += kLozBit[nb];
            }
    return t;
}

rt_status loz_extremal(const Vec& d, int dir, Vec* out) {
    const int m = isqrt_exact((int64_t)d.size() / 2);
    if (m < 2 || (int64_t)2 * m * m != (int64_t)d.size()) return RT_E_INVAL;
    const int n = m + 1;
    const Vec verts = loz_vertices(d, m);
    Vec hf((size_t)n * n, INF);
    const int start = first_boundary(verts);
    if (start < 0) return RT_E_INVAL;
    hf[start] = 0;
    std::deque<int> q{start};
    std::vector<int> seeds{start};
    while (!q.empty()) {
        const int v = q.front();
        q.pop_front();
        const int i = v / n, j = v % n;
        for (int nb = 0; nb < 6; ++nb) {
            const int i2 = i + kLozDi[nb], j2 = j + kLozDj[nb];
            if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n || verts[i2 * n + j2] != 2) continue;
            if (!loz_edge_in(d, m, i, j, nb, true)) continue;
            const int w = i2 * n + j2;
            const int32_t h = hf[v] + kLozDh[nb];
            if (hf[w] == INF) {
                hf[w] = h;
                q.push_back(w);
                seeds.push_back(w);
            } else if (hf[w] != h) {
                return RT_E_INVAL;
            }
        }
    }
    auto nbrs = [&](int v, int* out6) {
        const int i = v / n, j = v % n;
        for (int nb = 0; nb < 6; ++nb) {
            const int i2 = i + kLozDi[nb], j2 = j + kLozDj[nb];
            out6[nb] = (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n) ? -1 : i2 * n + j2;
        }
        return 6;
    };
    auto allowed = [&](int, int nb) { return kLozDh[nb] == dir; };
    if (!extremal_flood(hf, verts, seeds, dir, nbrs, allowed)) return RT_E_INVAL;
    for (size_t k = 0; k < hf.size(); ++k)
        if (verts[k] == 0) hf[k] = INF;
    *out = loz_height_to_tiling(hf, d, n);
    return RT_OK;
}

// Change of coordinates of the rectangle-triangle hexagons
// (RectTriangleTiler.cpp:446-456): row i moves down 3 and right N+3-i.
Vec rt_shear(const Vec& g, int n, int m) {
    const int m2 = m + 6 + (3 - m % 3) % 3;
    Vec out((size_t)m2 * m2, 0);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            const int j2 = j + n + 3 - i;
            if (j2 >= 0 && j2 < m2) out[(size_t)(i + 3) * m2 + j2] = g[(size_t)i * m + j];
        }
    return out;
}

}  // namespace

extern "C" {

// ---- dominoes ----------------------------------------------------------------
rt_status rt_domino_rectangle(int32_t rows, int32_t cols, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (rows < 0 || cols < 0 || std::max<int64_t>(rows, cols) + 5 > kMaxSide) return RT_E_INVAL;
        int dim = std::max(rows, cols) + 4;
        if (dim % 2 == 0) ++dim;
        Vec d((size_t)dim * dim, 0);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j) d[(size_t)(i + 2) * dim + j + 2] = 1;
        return emit(d, out, cap, len);
    });
}

rt_status rt_domino_aztec_rectangle(int32_t order, const int32_t* remove, int32_t k, int32_t* out, int64_t cap,
                                    int64_t* len) {
    return guarded([&]() -> rt_status {
        if (order < 1 || order > (kMaxSide - 5) / 2 || k < 0 || k >= 2 * order) return RT_E_INVAL;
        const int n = order, m = 2 * n - k;
        Vec d((size_t)m * m, 0);
        for (int i = 0; i < m; ++i) {
            int lo, hi;
            if (i == 0 || i == m - 1) {
                lo = (n - k) + (i == m - 1) * k - 1;
                hi = lo + 1;
            } else if (i < n - k) {
                lo = n - k - i - 1, hi = n - k + i;
            } else if (i > n - 1) {
                lo = i - n + k, hi = 3 * n - k - i - 1;
            } else {
                lo = i - (n - k), hi = i + (n - k);
            }
            for (int j = std::max(lo, 0); j <= std::min(hi, m - 1); ++j) d[(size_t)i * m + j] = 1;
        }
        for (int r = 0; r < k; ++r) {
            const int i0 = n - k + remove[r], j0 = remove[r];
            if (i0 < 0 || j0 < 0 || i0 >= m || j0 >= m) return RT_E_INVAL;
            d[(size_t)i0 * m + j0] = 0;
        }
        const int m2 = m + 4 + (1 - m % 2);  // odd side -> even tiling side (DominoTiler.cpp:183-184)
        Vec d2((size_t)m2 * m2, 0);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) d2[(size_t)(i + 2) * m2 + j + 2] = d[(size_t)i * m + j];
        return emit(d2, out, cap, len);
    });
}

rt_status rt_domino_aztec(int32_t order, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        return rt_domino_aztec_rectangle(order, nullptr, 0, out, cap, len);
    });
}

rt_status rt_domino_domain_to_vertices(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int m = isqrt_exact(dlen);
        if (!d || m < 1) return RT_E_INVAL;
        if (!out) return size_only((int64_t)(m + 1) * (m + 1), len);
        return emit(dom_vertices(Vec(d, d + dlen), m), out, cap, len);
    });
}

rt_status rt_domino_max_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (!d) return RT_E_INVAL;
        if (!out) return dom_side_query(dlen, len);
        Vec t;
        rt_status s = dom_extremal(Vec(d, d + dlen), +1, &t);
        return s != RT_OK ? s : emit(t, out, cap, len);
    });
}

rt_status rt_domino_min_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (!d) return RT_E_INVAL;
        if (!out) return dom_side_query(dlen, len);
        Vec t;
        rt_status s = dom_extremal(Vec(d, d + dlen), -1, &t);
        return s != RT_OK ? s : emit(t, out, cap, len);
    });
}

rt_status rt_domino_height_to_tiling(const int32_t* h, int64_t hlen, const int32_t* d, int64_t dlen, int32_t* out,
                                     int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(hlen);
        if (!h || !d || n < 2 || (int64_t)(n - 1) * (n - 1) != dlen) return RT_E_INVAL;
        if (!out) return size_only(hlen, len);
        return emit(dom_height_to_tiling(Vec(h, h + hlen), Vec(d, d + dlen), n), out, cap, len);
    });
}

rt_status rt_domino_tiling_to_height(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, int32_t* out,
                                     int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || !d || n < 2 || (int64_t)(n - 1) * (n - 1) != dlen) return RT_E_INVAL;
        if (!out) return size_only(tlen, len);
        const int m = n - 1;
        const Vec D(d, d + dlen);
        const Vec verts = dom_vertices(D, m);
        Vec hf((size_t)n * n, INF);
        const int start = first_boundary(verts);
        if (start >= 0) {
            hf[start] = 0;
            std::deque<int> q{start};
            while (!q.empty()) {
                const int v = q.front();
                q.pop_front();
                const int i = v / n, j = v % n;
                for (int nb = 0; nb < 4; ++nb) {
                    if (t[v] & kDomBit[nb]) continue;  // a domino crosses this edge
                    const int i2 = i + kDomDi[nb], j2 = j + kDomDj[nb];
                    if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n) continue;
                    const int w = i2 * n + j2;
                    if (verts[w] == 0 || hf[w] != INF) continue;
                    int f[4];
                    dom_edge_faces(i, j, nb, f);
                    if (!dom_face(D, m, f[0], f[1]) && !dom_face(D, m, f[2], f[3])) continue;
                    hf[w] = hf[v] + dom_dh(i, j, nb);
                    q.push_back(w);
                }
            }
        }
        return emit(hf, out, cap, len);
    });
}

rt_status rt_domino_tiling_to_domain(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || n < 2) return RT_E_INVAL;
        const int m = n - 1;
        Vec d((size_t)m * m, 0);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                if ((t[i * n + j] & (2 + 8)) || (t[(i + 1) * n + j + 1] & (1 + 4))) d[(size_t)i * m + j] = 1;
        return emit(d, out, cap, len);
    });
}

// ---- lozenges ------------------------------------------------------------------
rt_status rt_lozenge_almost_hex(int32_t side, int32_t cut, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (side < 1 || side > (kMaxSide - 9) / 2 || cut < 0 || cut > side) return RT_E_INVAL;
        const int n = side;
        const int rows = 2 * n, cols = 4 * n;
        Vec d((size_t)rows * cols, 0);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j)
                d[(size_t)i * cols + j] = i < n ? (2 * i + j - 1 >= 2 * n - 2) : (2 * i + j <= 6 * n - 2);
        for (int i = 0; i < cut; ++i)
            for (int j = cols - 2 * cut; j < cols; ++j) d[(size_t)i * cols + j] = 0;
        // 3 rows / 6 triangles of padding, then grow to a vertex side divisible by 3
        // (LozengeTiler.cpp:370-388).
        const int m2 = rows + 6;
        const int k = (3 - (m2 + 1) % 3) % 3;
        const int m3 = m2 + k;
        Vec d3((size_t)m3 * 2 * m3, 0);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j) d3[(size_t)(i + 3) * 2 * m3 + j + 6] = d[(size_t)i * cols + j];
        return emit(d3, out, cap, len);
    });
}

// Hexagon with sides a (top), b, c, a, b, c in the triangle-row encoding of
// AlmostHexDomain (LozengeTiler.cpp:344-388), which it generalises (a = b =
// c = N gives AlmostHexDomain(N, 0)): b + c rows of 2a + 2b triangles; row i
// starts at column max(0, 2b - 1 - 2i) (the upper-left side slants for b
// rows, the lower-left one is vertical for c rows) and ends at column
// 2a + 2b - 1 for i < c, then 2a + 2b - 2 - 2(i - c) (the upper-right side
// is vertical for c rows, the lower-right one slants for b rows).  The same
// padding as AlmostHexDomain follows.  No reference counterpart.
rt_status rt_lozenge_hexagon(int32_t a, int32_t b, int32_t c, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (a < 1 || b < 1 || c < 1 || (int64_t)b + c + 8 > kMaxSide || (int64_t)a + b + 9 > kMaxSide)
            return RT_E_INVAL;
        const int rows = b + c, cols = 2 * a + 2 * b;
        Vec d((size_t)rows * cols, 0);
        for (int i = 0; i < rows; ++i) {
            const int lo = std::max(0, 2 * b - 1 - 2 * i);
            const int hi = i < c ? 2 * a + 2 * b - 1 : 2 * a + 2 * b - 2 - 2 * (i - c);
            for (int j = lo; j <= hi && j < cols; ++j) d[(size_t)i * cols + j] = 1;
        }
        // 3 rows / 6 triangles of padding, then a square array of side m3
        // (vertex side divisible by 3) as LozengeTiler.cpp:370-388 builds it.
        const int m2 = std::max(rows + 6, (cols + 12 + 1) / 2);
        const int k = (3 - (m2 + 1) % 3) % 3;
        const int m3 = m2 + k;
        Vec d3((size_t)m3 * 2 * m3, 0);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j) d3[(size_t)(i + 3) * 2 * m3 + j + 6] = d[(size_t)i * cols + j];
        return emit(d3, out, cap, len);
    });
}

rt_status rt_lozenge_domain_to_vertices(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int m = isqrt_exact(dlen / 2);
        if (!d || m < 2 || (int64_t)2 * m * m != dlen) return RT_E_INVAL;
        if (!out) return size_only((int64_t)(m + 1) * (m + 1), len);
        return emit(loz_vertices(Vec(d, d + dlen), m), out, cap, len);
    });
}

rt_status rt_lozenge_max_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (!d) return RT_E_INVAL;
        if (!out) return loz_side_query(dlen, len);
        Vec t;
        rt_status s = loz_extremal(Vec(d, d + dlen), +1, &t);
        return s != RT_OK ? s : emit(t, out, cap, len);
    });
}

rt_status rt_lozenge_min_tiling(const int32_t* d, int64_t dlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (!d) return RT_E_INVAL;
        if (!out) return loz_side_query(dlen, len);
        Vec t;
        rt_status s = loz_extremal(Vec(d, d + dlen), -1, &t);
        return s != RT_OK ? s : emit(t, out, cap, len);
    });
}

rt_status rt_lozenge_height_to_tiling(const int32_t* h, int64_t hlen, const int32_t* d, int64_t dlen, int32_t* out,
                                      int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(hlen);
        if (!h || !d || n < 3 || (int64_t)2 * (n - 1) * (n - 1) != dlen) return RT_E_INVAL;
        if (!out) return size_only(hlen, len);
        return emit(loz_height_to_tiling(Vec(h, h + hlen), Vec(d, d + dlen), n), out, cap, len);
    });
}

rt_status rt_lozenge_tiling_to_height(const int32_t* t, int64_t tlen, const int32_t* d, int64_t dlen, int32_t* out,
                                      int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || !d || n < 3 || (int64_t)2 * (n - 1) * (n - 1) != dlen) return RT_E_INVAL;
        if (!out) return size_only(tlen, len);
        const int m = n - 1;
        const Vec D(d, d + dlen);
        const Vec verts = loz_vertices(D, m);
        Vec hf((size_t)n * n, INF);
        const int start = first_boundary(verts);
        if (start >= 0) {
            hf[start] = 0;
            std::deque<int> q{start};
            while (!q.empty()) {
                const int v = q.front();
                q.pop_front();
                const int i = v / n, j = v % n;
                for (int nb = 0; nb < 6; ++nb) {
                    if (t[v] & kLozBit[nb]) continue;  // a lozenge covers this edge
                    const int i2 = i + kLozDi[nb], j2 = j + kLozDj[nb];
                    if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n) continue;
                    const int w = i2 * n + j2;
                    if (verts[w] == 0 || hf[w] != INF || !loz_edge_in(D, m, i, j, nb, false)) continue;
                    hf[w] = hf[v] + kLozDh[nb];
                    q.push_back(w);
                }
            }
        }
        return emit(hf, out, cap, len);
    });
}

rt_status rt_lozenge_tiling_to_domain(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || n < 3) return RT_E_INVAL;
        const int m = n - 1;
        Vec d((size_t)2 * m * m, 0);
        auto set = [&](int r, int c) {
            if (r >= 0 && r < m && c >= 0 && c < 2 * m) d[(size_t)r * 2 * m + c] = 1;
        };
        for (int i = 0; i < n - 1; ++i)
            for (int j = 0; j < n - 1; ++j) {
                const int v = t[i * n + j];
                if (v & 1) set(i - 1, 2 * j), set(i - 1, 2 * j - 1);
                if (v & 2) set(i - 1, 2 * j), set(i - 1, 2 * j + 1);
                if (v & 8) set(i - 1, 2 * j + 1), set(i, 2 * j);
            }
        return emit(d, out, cap, len);
    });
}

// ---- rectangle-triangle hexagons -------------------------------------------------
rt_status rt_recttri_max_hex(int32_t side, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (side < 1 || side > (kMaxSide - 9) / 2) return RT_E_INVAL;
        const int n = side, m = 2 * n + 1;
        Vec g((size_t)m * m, 0);
        auto at = [&](int i, int j) -> int32_t& { return g[(size_t)i * m + j]; };
        for (int i = 1; i < m - 1; ++i)
            for (int j = 0; j < m; ++j) {
                int32_t v;
                if (j - i > n || i - j > n) v = 0;
                else if (i < n && j < n) v = 0x333333;
                else if (i < j && j > n) v = 0x111111;
                else if (i > n && i > j) v = 0x222222;
                else if (i == n && j < n) v = 0x333222;
                else if (i < n && j == n) v = 0x331311;
                else if (i == j && i > n) v = 0x211221;
                else v = 0x331221;  // the centre, i == j == n
                at(i, j) = v;
            }
        for (int i = 1; i < n; ++i) at(i, 0) = 0x003033, at(0, i) = 0x000333;
        for (int i = n + 1; i < m - 1; ++i) at(i, m - 1) = 0x110100, at(m - 1, i) = 0x222000;
        for (int i = 1; i < n; ++i) at(i, i + n) = 0x100110, at(i + n, i) = 0x022002;
        at(0, 0) = 0x000033;
        at(n, 0) = 0x003002;
        at(0, n) = 0x000310;
        at(m - 1, m - 1) = 0x210000;
        at(n, m - 1) = 0x100100;
        at(m - 1, n) = 0x022000;
        return emit(rt_shear(g, n, m), out, cap, len);
    });
}

rt_status rt_recttri_min_hex(int32_t side, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        if (side < 1 || side > (kMaxSide - 9) / 2) return RT_E_INVAL;
        const int n = side, m = 2 * n + 1;
        Vec g((size_t)m * m, 0);
        auto at = [&](int i, int j) -> int32_t& { return g[(size_t)i * m + j]; };
        for (int i = 1; i < m - 1; ++i)
            for (int j = 1; j < m - 1; ++j) {
                int32_t v;
                if (j - i > n || i - j > n) v = 0;
                else if (i > n && j > n) v = 0x333333;
                else if (i > j && j < n) v = 0x111111;
                else if (i < n && i < j) v = 0x222222;
                else if (i == n && j > n) v = 0x222333;
                else if (i > n && j == n) v = 0x113133;
                else if (i == j && i < n) v = 0x122112;
                else v = 0x122133;  // the centre
                at(i, j) = v;
            }
        for (int i = 1; i < n; ++i) at(i, 0) = 0x001011, at(0, i) = 0x000222;
        for (int i = n + 1; i < m - 1; ++i) at(i, m - 1) = 0x330300, at(m - 1, i) = 0x333000;
        for (int i = 1; i < n; ++i) at(i, i + n) = 0x200220, at(i + n, i) = 0x011001;
        at(0, 0) = 0x000012;
        at(m - 1, n) = 0x013000;
        at(n, m - 1) = 0x200300;
        at(0, n) = 0x000220;
        at(n, 0) = 0x001001;
        at(m - 1, m - 1) = 0x330000;
        return emit(rt_shear(g, n, m), out, cap, len);
    });
}

// LozengeToRectTriangle (RectTriangleTiler.cpp:523-565): each triangle of the
// lozenge domain becomes a rect-triangle face digit (1, 2 or 3 by the lozenge
// covering it) on its three corner vertices.
rt_status rt_recttri_from_lozenge(const int32_t* tl, int64_t tlen, const int32_t* dl, int64_t dlen, int32_t* out,
                                  int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen), m = isqrt_exact(dlen / 2);
        if (!tl || !dl || n < 2 || m < 1 || (int64_t)2 * m * m != dlen || m + 1 > n) return RT_E_INVAL;
        Vec t((size_t)n * n, 0);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < 2 * m; ++j) {
                if (dl[(size_t)i * 2 * m + j] != 1) continue;
                const int c = j / 2;
                if (j % 2 == 0) {  // downward-pointing face: corners (i, c), (i, c+1), (i+1, c)
                    const int v = tl[(size_t)i * n + c];
                    const int dgt = (v & 8) ? 1 : (v & 32) ? 3 : 2;
                    t[(size_t)i * n + c] += dgt;
                    t[(size_t)i * n + c + 1] += dgt << 8;
                    t[(size_t)(i + 1) * n + c] += dgt << 16;
                } else {  // upward face: corners (i, c+1), (i+1, c), (i+1, c+1)
                    const int v = tl[(size_t)i * n + c + 1];
                    const int dgt = (v & 16) ? 2 : (v & 32) ? 3 : 1;
                    t[(size_t)i * n + c + 1] += dgt << 4;
                    t[(size_t)(i + 1) * n + c] += dgt << 12;
                    t[(size_t)(i + 1) * n + c + 1] += dgt << 20;
                }
            }
        return emit(t, out, cap, len);
    });
}

// ---- dimers on the triangular lattice -------------------------------------------
// Tile state encoding of src/TriangleDimer/TriangleDimerTiler.h:13-67: the
// N x N "tiling" holds, at (even i, odd j) / (odd i, even j) / (odd i, odd j),
// the 4-bit lozenge states of the H / L / R edges of the triangular lattice.

// Tile states from edge indicator arrays h, l, r of eSize x eSize
// (IceCreamCone / TestButterfly, TriangleDimerTiler.cpp:281-296, :365-380).
static Vec td_tiles_from_edges(const Vec& h, const Vec& l, const Vec& r, int e) {
    const int ts = 2 * e;
    Vec t((size_t)ts * ts, 0);
    auto H = [&](int i, int j) { return h[(size_t)i * e + j]; };
    auto L = [&](int i, int j) { return l[(size_t)i * e + j]; };
    auto R = [&](int i, int j) { return r[(size_t)i * e + j]; };
    for (int i = 3; i < ts - 1; ++i)
        for (int j = 3; j < ts - 1; ++j) {
            int32_t v;
            if (i % 2 == 0) {
                if (j % 2 == 0) continue;
                v = R(i / 2 - 1, j / 2) + 2 * L(i / 2 - 1, j / 2 + 1) + 4 * R(i / 2, j / 2) + 8 * L(i / 2, j / 2);
            } else if (j % 2 == 0) {
                v = H(i / 2, j / 2) + 2 * R(i / 2, j / 2) + 4 * H(i / 2 + 1, j / 2 - 1) + 8 * R(i / 2, j / 2 - 1);
            } else {
                v = H(i / 2, j / 2) + 2 * L(i / 2, j / 2 + 1) + 4 * H(i / 2 + 1, j / 2) + 8 * L(i / 2, j / 2);
            }
            t[(size_t)i * ts + j] = v;
        }
    return t;
}

rt_status rt_tridimer_ice_cream_cone(int32_t side, int32_t cut, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        // A downward equilateral triangle of side N with a triangle of side M cut
        // from its top-left corner, as a dimer cover built row by row
        // (TriangleDimerTiler.cpp:236-332).  Parities the reference only warns
        // about are accepted (its construction then covers a slightly different
        // domain); cut > side - 1 is rejected.
        if (side < 1 || side > (kMaxSide - 8) / 2 || cut < 0 || cut > side - 1) return RT_E_INVAL;
        const int n = side, m = cut, e = n + 4;
        const int k = ((n + 1) * (n + 2) / 2) % 2;
        Vec h((size_t)e * e, 0), l((size_t)e * e, 0), r((size_t)e * e, 0);
        for (int i = 2; i < e - 2; ++i)
            for (int j = 2; j < e - i; ++j) {
                const size_t at = (size_t)i * e + j;
                if (i < m + 2) {
                    if ((i + j) % 2 == m % 2 && m != 0 && j > m + 3 - i) h[at] = 1;
                    if ((n - m) % 2 == 0 && i % 2 == 0 && j == e - i - 1) r[at] = 1;
                } else {
                    if (j % 2 == 0) h[at] = 1;
                    if (i % 4 == (3 + n % 2 + 2 * k) % 4 && j == e - i - 1) h[at] = 0, l[at] = 1;
                    if (i % 4 == (2 + n % 2 + 2 * k) % 4 && j == e - i - 1) r[at] = 1;
                }
            }
        return emit(td_tiles_from_edges(h, l, r, e), out, cap, len);
    });
}

rt_status rt_tridimer_hexagon(int32_t side, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        // Edges in the encoding of the IceCreamCone builder: h(i, j) joins (i, j)
        // and (i, j+1), l(i, j) joins (i, j) and (i+1, j), r(i, j) joins (i, j+1)
        // and (i+1, j) (the neighbours TilingToVertices reads, :711-737).
        if (side < 1 || side > 4096) return RT_E_INVAL;
        const int s = side, e = 2 * s + 8, off = 3;
        Vec h((size_t)e * e, 0), l((size_t)e * e, 0), r((size_t)e * e, 0);
        auto lo_y = [&](int x) { return std::max(0, s - x) + (x == 0 ? 1 : 0); };  // corner (0, s) removed
        auto hi_y = [&](int x) { return std::min(2 * s, 3 * s - x); };
        auto at = [&](int x, int y) { return (size_t)(x + off) * e + (y + off); };
        // A row whose count of free vertices is odd pairs one end vertex with the
        // matching end of the next row: the right end unless the row above took
        // that one, then the left end -- so every row's free vertices stay one
        // run, paired horizontally from the left.
        int taken = 0;  // end of this row already paired with the row above: 0 none, 1 left, 2 right
        for (int x = 0; x <= 2 * s; ++x) {
            const int above = taken;
            int a = lo_y(x) + (above == 1), b = hi_y(x) - (above == 2);
            taken = 0;
            if ((b - a + 1) % 2 != 0) {
                if (x == 2 * s) return RT_E_STATE;  // unreachable: the vertex count is even
                if (above == 2) {
                    // left end (x, a) with the first vertex of the next row
                    const int t = lo_y(x + 1);
                    if (t == a) l[at(x, a)] = 1;
                    else if (t == a - 1) r[at(x, a - 1)] = 1;
                    else return RT_E_STATE;
                    taken = 1;
                    ++a;
                } else {
                    const int t = hi_y(x + 1);
                    if (t == b) l[at(x, b)] = 1;
                    else if (t == b - 1) r[at(x, b - 1)] = 1;
                    else return RT_E_STATE;
                    taken = 2;
                    --b;
                }
            }
            for (int y = a; y < b; y += 2) h[at(x, y)] = 1;
        }
        return emit(td_tiles_from_edges(h, l, r, e), out, cap, len);
    });
}

rt_status rt_tridimer_test_butterfly(int32_t kind, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        // One butterfly of orientation H (0), L (1) or R (2) (TriangleDimerTiler.cpp:334-383).
        if (kind < 0 || kind > 2) return RT_E_INVAL;
        const int e = 8;
        Vec h((size_t)e * e, 0), l((size_t)e * e, 0), r((size_t)e * e, 0);
        if (kind == 0) h[2 * e + 3] = h[4 * e + 3] = r[2 * e + 4] = r[3 * e + 2] = 1;
        if (kind == 1) r[2 * e + 3] = r[4 * e + 2] = l[3 * e + 2] = l[3 * e + 4] = 1;
        if (kind == 2) l[2 * e + 4] = l[4 * e + 3] = r[3 * e + 2] = r[3 * e + 4] = 1;
        return emit(td_tiles_from_edges(h, l, r, e), out, cap, len);
    });
}

}  // extern "C"

namespace rtb {
// Triangle-flip states ((N/2) x N) and butterfly-flip states (N x N) of a
// tiling (TilingToTriangleFlips / TilingToButterflyFlips,
// TriangleDimerTiler.cpp:385-460).
void td_derived_states(const int32_t* t, int n, int32_t* tri, int32_t* bfl) {
    auto T = [&](int i, int j) { return t[(size_t)i * n + j]; };
    std::fill(tri, tri + (size_t)(n / 2) * n, 0);
    std::fill(bfl, bfl + (size_t)n * n, 0);
    auto b = [](int32_t x, int k) { return (x >> k) & 1; };
    for (int i = 1; i < n / 2 - 1; ++i)
        for (int j = 1; j < n - 1; ++j) {
            const int32_t a = T(2 * i + 1, j), c = T(2 * i + 1, j + 1);
            int d0, d1, d2;
            if (j % 2 == 0) {  // down triangle
                const int32_t u = T(2 * i, j + 1);
                d0 = b(a, 2) + 2 * b(a, 3) + 3 * b(c, 3);
                d1 = b(c, 2) + 2 * b(a, 1) + 3 * b(c, 1);
                d2 = 2 * b(u, 0) + b(a, 0) + 3 * b(u, 1);
            } else {  // up triangle
                const int32_t w = T(2 * i + 2, j);
                d0 = b(a, 0) + 2 * b(a, 3) + 3 * b(c, 3);
                d1 = b(c, 0) + 2 * b(a, 1) + 3 * b(c, 1);
                d2 = 2 * b(w, 3) + 3 * b(w, 2) + b(a, 2);
            }
            tri[(size_t)i * n + j] = d0 + 4 * d1 + 16 * d2;
        }
    for (int i = 2; i < n - 2; ++i)
        for (int j = 2; j < n - 2; ++j) {
            const int32_t x = T(i, j);
            int f1, f4, f16, f64, c;
            if (i % 2 == 0) {
                if (j % 2 == 0) continue;
                const int32_t u = T(i - 1, j), ue = T(i - 1, j + 1), d = T(i + 1, j), dw = T(i + 1, j - 1);
                f1 = b(u, 3) + 2 * b(u, 0) + 3 * b(x, 0);
                f4 = b(ue, 0) + 2 * b(ue, 1) + 3 * b(x, 1);
                f16 = b(d, 1) + 2 * b(d, 2) + 3 * b(x, 2);
                f64 = b(dw, 2) + 2 * b(dw, 3) + 3 * b(x, 3);
                c = b(ue, 2);
            } else if (j % 2 == 0) {
                const int32_t ue = T(i - 1, j + 1), e = T(i, j + 1), dw = T(i + 1, j - 1), w = T(i, j - 1);
                f1 = b(ue, 0) + 2 * b(ue, 1) + 3 * b(x, 0);
                f4 = b(e, 1) + 2 * b(e, 2) + 3 * b(x, 1);
                f16 = b(dw, 2) + 2 * b(dw, 3) + 3 * b(x, 2);
                f64 = b(w, 3) + 2 * b(w, 0) + 3 * b(x, 3);
                c = b(e, 3);
            } else {
                const int32_t u = T(i - 1, j), e = T(i, j + 1), d = T(i + 1, j), w = T(i, j - 1);
                f1 = b(u, 0) + 2 * b(u, 1) + 3 * b(x, 0);
                f4 = b(e, 0) + 2 * b(e, 1) + 3 * b(x, 1);
                f16 = b(d, 2) + 2 * b(d, 3) + 3 * b(x, 2);
                f64 = b(w, 2) + 2 * b(w, 3) + 3 * b(x, 3);
                c = b(e, 3);
            }
            bfl[(size_t)i * n + j] = f1 + 4 * f4 + 16 * f16 + 64 * f64 + 256 * c;
        }
}

// The eight M x M arrays the walk runs on (TriangleDimerTiler.cpp:107-133),
// in the order H, L, R, U, D, BH, BL, BR.
void td_split_host(const int32_t* t, int n, int32_t* arrays) {
    const int m = n / 2;
    const size_t mm = (size_t)m * m;
    Vec tri((size_t)(n / 2) * n), bfl((size_t)n * n);
    td_derived_states(t, n, tri.data(), bfl.data());
    std::fill(arrays, arrays + 8 * mm, 0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const size_t at = (size_t)(i / 2) * m + j / 2;
            const size_t src = (size_t)i * n + j;
            if (i % 2 == 0) {
                if (j % 2 == 1) arrays[0 * mm + at] = t[src], arrays[5 * mm + at] = bfl[src];
            } else if (j % 2 == 0) {
                arrays[1 * mm + at] = t[src], arrays[6 * mm + at] = bfl[src];
            } else {
                arrays[2 * mm + at] = t[src], arrays[7 * mm + at] = bfl[src];
            }
        }
    for (int i = 0; i < n / 2; ++i)
        for (int j = 0; j < n; ++j) arrays[(j % 2 == 0 ? 4 : 3) * mm + (size_t)i * m + j / 2] = tri[(size_t)i * n + j];
}
}  // namespace rtb

extern "C" {

rt_status rt_tridimer_triangle_flips(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || n < 2 || n % 2) return RT_E_INVAL;
        Vec tri((size_t)(n / 2) * n), bfl((size_t)n * n);
        rtb::td_derived_states(t, n, tri.data(), bfl.data());
        return emit(tri, out, cap, len);
    });
}

rt_status rt_tridimer_butterfly_flips(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || n < 2 || n % 2) return RT_E_INVAL;
        Vec tri((size_t)(n / 2) * n), bfl((size_t)n * n);
        rtb::td_derived_states(t, n, tri.data(), bfl.data());
        return emit(bfl, out, cap, len);
    });
}

// Vertices covered by a dimer ((N/2+1)^2, TilingToVertices :711-737).
static Vec td_vertices(const int32_t* t, int n) {
    const int m = n / 2 + 1;
    Vec v((size_t)m * m, 0);
    for (int i = 2; i < m - 2; ++i)
        for (int j = 2; j < m - 2; ++j) {
            const int32_t a = t[(size_t)2 * (i - 1) * n + 2 * j + 1], b = t[(size_t)2 * (i + 1) * n + 2 * j - 1];
            const int32_t c = t[(size_t)(2 * i - 1) * n + 2 * j], d = t[(size_t)(2 * i - 1) * n + 2 * j + 1];
            v[(size_t)i * m + j] = ((a & 12) || (b & 3) || (c & 4) || (d & 4)) ? 1 : 0;
        }
    return v;
}

rt_status rt_tridimer_vertices(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || n < 8 || n % 2) return RT_E_INVAL;
        return emit(td_vertices(t, n), out, cap, len);
    });
}

// Triangles whose three corners are covered (TilingToDomain :739-770).
rt_status rt_tridimer_tiling_to_domain(const int32_t* t, int64_t tlen, int32_t* out, int64_t cap, int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || n < 8 || n % 2) return RT_E_INVAL;
        const int m = n / 2 + 1;
        const Vec v = td_vertices(t, n);
        Vec d((size_t)(m - 1) * 2 * (m - 1), 0);
        auto V = [&](int i, int j) { return v[(size_t)i * m + j] == 1; };
        for (int i = 0; i < m - 1; ++i)
            for (int j = 0; j < 2 * (m - 1); ++j) {
                const bool in = j % 2 == 0 ? (V(i, j / 2) && V(i, j / 2 + 1) && V(i + 1, j / 2))
                                           : (V(i, j / 2 + 1) && V(i + 1, j / 2) && V(i + 1, j / 2 + 1));
                d[(size_t)i * 2 * (m - 1) + j] = in;
            }
        return emit(d, out, cap, len);
    });
}

// 0/1 indicator of dimers of one orientation (DimerIndicator :20-84; the
// reference reads orientations 1 and 2 from the (even, odd) cells and 0 from
// the (odd, odd) cells, bits 8, 4 and 1 respectively).
rt_status rt_tridimer_dimer_indicator(const int32_t* t, int64_t tlen, int32_t orient, int32_t* out, int64_t cap,
                                      int64_t* len) {
    return guarded([&]() -> rt_status {
        const int n = isqrt_exact(tlen);
        if (!t || n < 2 || n % 2 || orient < 0 || orient > 2) return RT_E_INVAL;
        const int m = n / 2;
        Vec dd((size_t)m * m, 0);
        const int bit = orient == 1 ? 8 : orient == 2 ? 4 : 1;
        const int ri = orient == 0 ? 1 : 0;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                dd[(size_t)i * m + j] = (t[(size_t)(2 * i + ri) * n + 2 * j + 1] & bit) == bit;
        return emit(dd, out, cap, len);
    });
}

}  // extern "C"

extern "C" rt_status rt_mixed_chain_spec(int64_t seed, int32_t* model, int32_t* p) {
    if (!model || !p || seed < 0) return RT_E_INVAL;
    std::mt19937 mt((std::mt19937::result_type)seed);
    p[0] = p[1] = p[2] = 0;
    switch (seed % 4) {
        case 0: {
            std::uniform_int_distribution<int> n(16, 256);
            *model = RT_DOMINO;
            p[0] = n(mt);
            break;
        }
        case 1: {
            std::uniform_int_distribution<int> side(8, 128);
            *model = RT_LOZENGE;
            p[0] = side(mt);
            p[1] = side(mt);
            p[2] = side(mt);
            break;
        }
        case 2:  // bibone hexagon of side 64 (rt_tridimer_hexagon)
            *model = RT_TRIDIMER;
            p[0] = 64;
            break;
        default:
            *model = RT_RECTTRI;
            p[0] = 64;
            break;
    }
    return RT_OK;
}

namespace rtb {

// The graph the height-function projection relaxes over (rt_project.cu):
// vertex side *n, per vertex its kind (0 outside the domain, 1 interior,
// 2 boundary -- as DomainToVertices marks them) and a bit per neighbour
// direction whose edge touches the domain with both ends inside it.
// Directions: dominoes (i+1, j), (i-1, j), (i, j+1), (i, j-1); lozenges
// (i, j+1), (i-1, j+1), (i-1, j), (i, j-1), (i+1, j-1), (i+1, j).
bool lipschitz_graph(int model, const int32_t* d, int64_t dlen, int* n_out, std::vector<uint8_t>* kind,
                     std::vector<uint8_t>* edges) {
    if (!d) return false;
    if (model == RT_DOMINO) {
        const int m = isqrt_exact(dlen);
        if (m < 1) return false;
        const int n = m + 1;
        const Vec D(d, d + dlen);
        const Vec verts = dom_vertices(D, m);
        kind->assign((size_t)n * n, 0);
        edges->assign((size_t)n * n, 0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const int v = i * n + j;
                (*kind)[v] = (uint8_t)verts[v];
                if (!verts[v]) continue;
                for (int nb = 0; nb < 4; ++nb) {
                    const int i2 = i + kDomDi[nb], j2 = j + kDomDj[nb];
                    if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n || !verts[i2 * n + j2]) continue;
                    int f[4];
                    dom_edge_faces(i, j, nb, f);
                    if (dom_face(D, m, f[0], f[1]) || dom_face(D, m, f[2], f[3])) (*edges)[v] |= (uint8_t)(1u << nb);
                }
            }
        *n_out = n;
        return true;
    }
    if (model == RT_LOZENGE) {
        const int m = isqrt_exact(dlen / 2);
        if (m < 2 || (int64_t)2 * m * m != dlen) return false;
        const int n = m + 1;
        const Vec D(d, d + dlen);
        const Vec verts = loz_vertices(D, m);
        kind->assign((size_t)n * n, 0);
        edges->assign((size_t)n * n, 0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const int v = i * n + j;
                (*kind)[v] = (uint8_t)verts[v];
                if (!verts[v]) continue;
                for (int nb = 0; nb < 6; ++nb) {
                    const int i2 = i + kLozDi[nb], j2 = j + kLozDj[nb];
                    if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n || !verts[i2 * n + j2]) continue;
                    if (loz_edge_in(D, m, i, j, nb, false)) (*edges)[v] |= (uint8_t)(1u << nb);
                }
            }
        *n_out = n;
        return true;
    }
    return false;
}

// Heights of the boundary vertices reachable from the first boundary vertex
// (row-major, height 0) along boundary edges -- edges with the domain on one
// side only, which no tile crosses, so the height steps by the edge's
// orientation -- exactly as the first step of dom_extremal / loz_extremal
// (Thurston's construction, DominoTiler.cpp:214-399, LozengeTiler.cpp:140-318),
// but with vertex kinds computed on the fly: only the rows up to the first
// boundary vertex and the boundary itself are visited, never the whole
// N x N grid.  Returns false when the domain has no boundary vertex or the
// heights disagree around the boundary (not tileable).
bool boundary_walk(int model, const int32_t* d, int64_t dlen, int* n_out, std::vector<int64_t>* idx,
                   std::vector<int32_t>* h) {
    if (!d || (model != RT_DOMINO && model != RT_LOZENGE)) return false;
    const bool dom = model == RT_DOMINO;
    const int m = dom ? isqrt_exact(dlen) : isqrt_exact(dlen / 2);
    if (m < (dom ? 1 : 2) || (!dom && (int64_t)2 * m * m != dlen)) return false;
    const int n = m + 1;
    auto kind = [&](int i, int j) { return dom ? dom_vertex_kind(d, m, i, j) : loz_vertex_kind(d, m, i, j); };
    int64_t start = -1;
    for (int i = 0; i < n && start < 0; ++i)
        for (int j = 0; j < n; ++j)
            if (kind(i, j) == 2) {
                start = (int64_t)i * n + j;
                break;
            }
    if (start < 0) return false;
    std::unordered_map<int64_t, int32_t> hf;
    hf[start] = 0;
    idx->assign(1, start);
    h->assign(1, 0);
    for (size_t at = 0; at < idx->size(); ++at) {
        const int64_t v = (*idx)[at];
        const int i = (int)(v / n), j = (int)(v % n);
        const int32_t hv = (*h)[at];
        for (int nb = 0; nb < (dom ? 4 : 6); ++nb) {
            const int i2 = i + (dom ? kDomDi[nb] : kLozDi[nb]), j2 = j + (dom ? kDomDj[nb] : kLozDj[nb]);
            if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n || kind(i2, j2) != 2) continue;
            int32_t step;
            if (dom) {
                int f[4];
                dom_edge_faces(i, j, nb, f);
                if ((dom_face_p(d, m, f[0], f[1]) != 0) == (dom_face_p(d, m, f[2], f[3]) != 0)) continue;
                step = dom_dh(i, j, nb);
            } else {
                if (!loz_edge_in_p(d, m, i, j, nb, true)) continue;
                step = kLozDh[nb];
            }
            const int64_t w = (int64_t)i2 * n + j2;
            auto it = hf.find(w);
            if (it == hf.end()) {
                hf.emplace(w, hv + step);
                idx->push_back(w);
                h->push_back(hv + step);
            } else if (it->second != hv + step) {
                return false;
            }
        }
    }
    *n_out = n;
    return true;
}

}  // namespace rtb
