/* sixv_oracle.c -- CPU restatement of the six-vertex (square ice) dynamics.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA six-vertex walk.  The
 * reference names the six-vertex model (README.md:3) but ships no source for
 * it, so there is no reference code to replay; this file states the model
 * and its Glauber dynamics as this project defines them, and the tests pin it
 * against exact enumeration of the model on small domains.
 *
 * Model.  An n x n grid of vertices with domain-wall boundary conditions is a
 * height function h on the (n+1) x (n+1) faces: h(0,j) = j, h(i,0) = i,
 * h(n,j) = n-j, h(i,n) = n-i, faces sharing an edge differ by 1 (the corner
 * sums of an alternating-sign matrix: h = i + j - 2 sum_{k<=i,l<=j} A_kl).
 * The vertex (i,j), 1 <= i,j <= n, sits between the faces NW = (i-1,j-1),
 * NE = (i-1,j), SW = (i,j-1), SE = (i,j) with heights a, b, c, d; its type is
 *   0 (a1): b = a+1, c = a-1, d = a      1 (a2): b = a-1, c = a+1, d = a
 *   2 (b1): b = c = a+1, d = a+2         3 (b2): b = c = a-1, d = a-2
 *   4 (c1): b = c = a+1, d = a (A = +1)  5 (c2): b = c = a-1, d = a (A = -1)
 * and a configuration weighs the product of its vertices' type weights.
 *
 * Dynamics (heat bath).  An interior face (1 <= i,j <= n-1) whose four
 * edge neighbours share one height m holds m-1 or m+1; it is resampled with
 * P(m+1) = W(m+1) / (W(m+1) + W(m-1)), the product of the weights of its four
 * corner vertices, which depend on m, the face and its four diagonal
 * neighbours (each m-1 or m+1).  The host turns the 16 diagonal patterns into
 * integer thresholds on a 23-bit draw k: up iff k < ceil(P 2^23).  Faces are
 * coloured by (i mod 2, j mod 2); colour step s of an epoch updates class
 * s mod 4 (row parity (s mod 4) / 2, column parity s mod 2) -- faces of one
 * class share no neighbour, edge or diagonal -- and a sweep is four steps.
 *
 * Draws.  The faces (i, 8q + p + 2b), b = 0..3, of one row and column parity
 * p take output words b of Philox4x32-10(counter = (i Q + q, s lo, s hi,
 * chain), key = the epoch key), Q = ceil((n+1)/8); k = word >> 9.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "rt_oracle.h"

void orc_sixv_dwbc(int n, int32_t* hmin, int32_t* hmax) {
    for (int i = 0; i <= n; ++i)
        for (int j = 0; j <= n; ++j) {
            const int at = i * (n + 1) + j;
            if (hmin) hmin[at] = abs(i - j);
            if (hmax) hmax[at] = i + j < 2 * n - i - j ? i + j : 2 * n - i - j;
        }
}

int orc_sixv_vertex_type(int a, int b, int c, int d) {
    if (b == a + 1 && c == a - 1 && d == a) return 0;
    if (b == a - 1 && c == a + 1 && d == a) return 1;
    if (b == a + 1 && c == a + 1) return d == a + 2 ? 2 : d == a ? 4 : -1;
    if (b == a - 1 && c == a - 1) return d == a - 2 ? 3 : d == a ? 5 : -1;
    return -1;
}

/* Thresholds of the heat bath for the 16 diagonal patterns: bit 0 NW
 * (i-1,j-1), bit 1 NE (i-1,j+1), bit 2 SW (i+1,j-1), bit 3 SE (i+1,j+1) set
 * when that face is at m+1 (clear: m-1). */
void orc_sixv_thresholds(const double w[6], uint32_t thr[16]) {
    for (int p = 0; p < 16; ++p) {
        const int d1 = (p & 1) ? 1 : -1, d2 = (p & 2) ? 1 : -1, d3 = (p & 4) ? 1 : -1, d4 = (p & 8) ? 1 : -1;
        double wt[2];
        for (int up = 0; up < 2; ++up) {
            const int h = up ? 1 : -1; /* heights relative to m */
            const int t1 = orc_sixv_vertex_type(d1, 0, 0, h);  /* vertex (i, j):     NW d1, NE m, SW m, SE h */
            const int t2 = orc_sixv_vertex_type(0, d2, h, 0);  /* vertex (i, j+1):   NW m, NE d2, SW h, SE m */
            const int t3 = orc_sixv_vertex_type(0, h, d3, 0);  /* vertex (i+1, j):   NW m, NE h, SW d3, SE m */
            const int t4 = orc_sixv_vertex_type(h, 0, 0, d4);  /* vertex (i+1, j+1): NW h, NE m, SW m, SE d4 */
            wt[up] = w[t1] * w[t2] * w[t3] * w[t4];
        }
        const double s = ceil(wt[1] / (wt[0] + wt[1]) * 8388608.0);
        thr[p] = s <= 0 ? 0u : s >= 4294967295.0 ? 0xffffffffu : (uint32_t)s;
    }
}

/* Colour step s on the face rows i in [lo, hi) only (the whole step is
 * lo = 1, hi = n). */
static void sixv_step_range(int32_t* h, int n, int64_t s, uint64_t key, uint32_t chain, const uint32_t thr[16],
                            int lo, int hi) {
    const int N1 = n + 1, Q = (N1 + 7) / 8;
    const int pi = (int)((s & 3) >> 1), pj = (int)(s & 1);
    const uint32_t k2[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
    int first = pi == 0 ? 2 : 1;
    if (lo > first) first += ((lo - first + 1) / 2) * 2;
    if (hi > n) hi = n;
    for (int i = first; i < hi; i += 2)
        for (int q = 0; q < Q; ++q) {
            const uint32_t ctr[4] = {(uint32_t)(i * Q + q), (uint32_t)s, (uint32_t)((uint64_t)s >> 32), chain};
            uint32_t out[4];
            orc_philox4x32_10(ctr, k2, out);
            for (int b = 0; b < 4; ++b) {
                const int j = 8 * q + pj + 2 * b;
                if (j < 1 || j > n - 1) continue;
                int32_t* f = &h[i * N1 + j];
                const int m = f[-N1];
                if (f[N1] != m || f[-1] != m || f[1] != m) continue;
                const int p = (f[-N1 - 1] > m) | ((f[-N1 + 1] > m) << 1) | ((f[N1 - 1] > m) << 2) | ((f[N1 + 1] > m) << 3);
                *f = (out[b] >> 9) < thr[p] ? m + 1 : m - 1;
            }
        }
}

static void sixv_step(int32_t* h, int n, int64_t s, uint64_t key, uint32_t chain, const uint32_t thr[16]) {
    sixv_step_range(h, n, s, key, chain, thr, 1, n);
}

int orc_sixv_step_rows(int32_t* h, int n, int64_t s, uint64_t key, uint32_t chain, const double w[6], int lo,
                       int hi) {
    if (n < 1 || !h || !w || s < 0) return ORC_EINVAL;
    for (int t = 0; t < 6; ++t)
        if (!(w[t] > 0) || !isfinite(w[t])) return ORC_EINVAL;
    uint32_t thr[16];
    orc_sixv_thresholds(w, thr);
    sixv_step_range(h, n, s, key, chain, thr, lo, hi);
    return ORC_OK;
}

int orc_sixv_walk(int32_t* h, int n, const int64_t* sweeps, const int64_t* keys, int k, uint32_t chain,
                  const double w[6]) {
    if (n < 1 || k < 0 || !h || !w) return ORC_EINVAL;
    for (int t = 0; t < 6; ++t)
        if (!(w[t] > 0) || !isfinite(w[t])) return ORC_EINVAL;
    uint32_t thr[16];
    orc_sixv_thresholds(w, thr);
    for (int e = 0; e < k; ++e) {
        if (sweeps[e] < 0) return ORC_EINVAL;
        for (int64_t s = 0; s < 4 * sweeps[e]; ++s) sixv_step(h, n, s, (uint64_t)keys[e], chain, thr);
    }
    return ORC_OK;
}
