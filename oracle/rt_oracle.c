/* rt_oracle.c -- CPU restatement of RandomTilings' flip dynamics (the checker).
 *
 * TEST INFRASTRUCTURE ONLY; see rt_oracle.h.  Every function below restates
 * one piece of the reference and cites it; the restatement is pinned against
 * the reference's own code run on the CPU (oracle/_ref) by the tests.
 *
 * The reference runs each colour step as OpenCL kernels whose work items are
 * independent (each writes only its own site of arrays it does not read at
 * other sites), so a serial loop over the NDRange reproduces the device
 * result exactly; that is how the kernels are restated here.
 */
#include "rt_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* TinyMT32 (Saito & Matsumoto), as used per work item by the reference:    */
/* src/TinyMT/tinymt32.clh:39-55 (next_state), :81-93 (temper12),          */
/* :125-129 (single01), :182-203 (init).                                    */
/* ------------------------------------------------------------------------ */
#define TMT_J_MAT1 0x8f7011eeu /* src/TinyMT/tinymt32def.h:47-49 */
#define TMT_J_MAT2 0xfc78ff1fu
#define TMT_J_TMAT 0x3793fdffu

static void tmt_step(orc_tinymt* s) {
    uint32_t x = (s->s0 & 0x7fffffffu) ^ s->s1 ^ s->s2;
    uint32_t y = s->s3;
    x ^= x << 1;
    y ^= (y >> 1) ^ x;
    s->s0 = s->s1;
    s->s1 = s->s2;
    s->s2 = x ^ (y << 10);
    s->s3 = y;
    if (y & 1u) {
        s->s1 ^= s->mat1;
        s->s2 ^= s->mat2;
    }
}

static uint32_t tmt_temper(const orc_tinymt* s) {
    uint32_t t1 = s->s0 + (s->s2 >> 8);
    uint32_t t0 = s->s3 ^ t1;
    if (t1 & 1u) t0 ^= s->tmat;
    return t0;
}

void orc_tinymt_init(orc_tinymt* st, uint32_t seed) {
    uint32_t v[4] = {seed, st->mat1, st->mat2, st->tmat};
    for (int i = 1; i < 8; ++i) {
        uint32_t p = v[(i - 1) & 3];
        v[i & 3] ^= (uint32_t)i + 1812433253u * (p ^ (p >> 30));
    }
    st->s0 = v[0];
    st->s1 = v[1];
    st->s2 = v[2];
    st->s3 = v[3];
    if ((st->s0 & 0x7fffffffu) == 0 && st->s1 == 0 && st->s2 == 0 && st->s3 == 0) {
        st->s0 = 'T';
        st->s1 = 'I';
        st->s2 = 'N';
        st->s3 = 'Y';
    }
    for (int i = 0; i < 8; ++i) {
        tmt_step(st);
        (void)tmt_temper(st);
    }
}

uint32_t orc_tinymt_bits12(orc_tinymt* st) {
    tmt_step(st);
    return (tmt_temper(st) >> 9) | 0x3f800000u;
}

float orc_tinymt_single01(orc_tinymt* st) {
    uint32_t b = orc_tinymt_bits12(st);
    float f;
    memcpy(&f, &b, sizeof f);
    return f - 1.0f;
}

/* Per-work-item generators seeded as InitTinyMT does: stream `id` starts
 * from init(seed + id) with the id-th parameter triple (e.g.
 * src/Domino/dominokernel.cl:33-40, src/TinyMT/file_reader.cpp:22-38). */
static orc_tinymt* tmt_streams(int64_t count, uint32_t seed, const uint32_t* params, int64_t nparams, int* err) {
    if (params && nparams < count) {
        *err = ORC_EPARAMS;
        return NULL;
    }
    orc_tinymt* s = (orc_tinymt*)malloc((size_t)(count > 0 ? count : 1) * sizeof *s);
    if (!s) {
        *err = ORC_ENOMEM;
        return NULL;
    }
    for (int64_t id = 0; id < count; ++id) {
        s[id].mat1 = params ? params[3 * id + 0] : TMT_J_MAT1;
        s[id].mat2 = params ? params[3 * id + 1] : TMT_J_MAT2;
        s[id].tmat = params ? params[3 * id + 2] : TMT_J_TMAT;
        orc_tinymt_init(&s[id], seed + (uint32_t)id);
    }
    *err = ORC_OK;
    return s;
}

/* ------------------------------------------------------------------------ */
/* Host colour generators.                                                  */
/* std::mt19937 (DominoTiler.cpp:31,35,81,85): the standard MT19937.        */
/* std::default_random_engine is libstdc++'s minstd_rand0 (a = 16807,       */
/* m = 2^31-1); std::uniform_int_distribution<int>(0, hi) maps one engine   */
/* output through libstdc++'s rejection + division downscaling             */
/* (LozengeTiler.cpp:50-55, RectTriangleTiler.cpp:41-48,                    */
/* TriangleDimerTiler.cpp:230-241).                                         */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint32_t v[624];
    int pos;
} mt_state;

static void mt_seed(mt_state* m, int64_t seed) {
    m->v[0] = (uint32_t)(uint64_t)seed; /* result_type seed, reduced mod 2^32 */
    for (int i = 1; i < 624; ++i) m->v[i] = 1812433253u * (m->v[i - 1] ^ (m->v[i - 1] >> 30)) + (uint32_t)i;
    m->pos = 624;
}

static uint32_t mt_next(mt_state* m) {
    if (m->pos >= 624) {
        for (int k = 0; k < 624; ++k) {
            uint32_t y = (m->v[k] & 0x80000000u) | (m->v[(k + 1) % 624] & 0x7fffffffu);
            m->v[k] = m->v[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        m->pos = 0;
    }
    uint32_t y = m->v[m->pos++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

void orc_mt19937_stream(int64_t seed, int64_t n, uint32_t* out) {
    mt_state m;
    mt_seed(&m, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = mt_next(&m);
}

typedef struct {
    uint64_t x;
} minstd;

static void minstd_seed(minstd* g, int64_t seed) {
    g->x = ((uint64_t)seed) % 2147483647u; /* seed is taken as an unsigned 64-bit result_type */
    if (g->x == 0) g->x = 1;
}

static uint32_t minstd_next(minstd* g) {
    g->x = (g->x * 16807u) % 2147483647u;
    return (uint32_t)g->x;
}

static int uniform_int(minstd* g, int hi) {
    const uint64_t range = 2147483646u - 1u; /* engine max - min */
    const uint64_t buckets = (uint64_t)hi + 1u;
    const uint64_t scale = range / buckets;
    const uint64_t limit = buckets * scale;
    uint64_t r;
    do {
        r = (uint64_t)minstd_next(g) - 1u;
    } while (r >= limit);
    return (int)(r / scale);
}

void orc_minstd_raw_stream(int64_t seed, int64_t n, uint32_t* out) {
    minstd g;
    minstd_seed(&g, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = minstd_next(&g);
}

void orc_minstd_uniform_stream(int64_t seed, int64_t n, const int* his, int nhis, int* out) {
    minstd g;
    minstd_seed(&g, seed);
    for (int64_t i = 0; i < n; ++i) out[i] = uniform_int(&g, his[i % nhis]);
}

/* Colour choice of every step of a Walk. */
int orc_domino_colours(int64_t seed, int64_t steps, int single_walk, uint8_t* out) {
    mt_state m;
    mt_seed(&m, seed);
    if (single_walk) (void)mt_next(&m); /* first output seeds TinyMT, DominoTiler.cpp:31-32 */
    for (int64_t i = 0; i < steps; ++i) out[i] = (uint8_t)(mt_next(&m) % 2u);
    return ORC_OK;
}

int orc_lozenge_colours(int64_t seed, int64_t steps, uint8_t* out) {
    minstd g;
    minstd_seed(&g, seed);
    for (int64_t i = 0; i < steps; ++i) out[i] = (uint8_t)uniform_int(&g, 2);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Domino: src/Domino/DominoTiler.cpp:9-107, dominokernel.cl, and           */
/* dominokernelCFTP.cl.  Vertex state bits: 1 up, 2 down, 8 towards j+1,   */
/* 4 towards j-1 (the order DominoTiler.cpp:204-206 uses).  Black vertices  */
/* ((i+j) even) and white ones live in separate N x N/2 byte arrays.        */
/* ------------------------------------------------------------------------ */
/* RotateTiles, dominokernel.cl:4-18 (flip 3<->12 when rd < .8) and
 * dominokernelCFTP.cl:11-31 (heat bath: rd < .5 -> 12, else -> 3).
 * Work item (g0, g1) of the (N-2) x (N/2-2) range owns site (g0+1, g1+1) and
 * TinyMT stream g1 + (N/2-2) g0 (src/TinyMT/tinymt.clh:24-30). */
static void domino_rotate(int8_t* a, int n, orc_tinymt* rng, int cftp) {
    const int h = n / 2, gw = h - 2;
    for (int g0 = 0; g0 < n - 2; ++g0)
        for (int g1 = 0; g1 < gw; ++g1) {
            const int64_t id = (int64_t)g1 + (int64_t)gw * g0;
            const float rd = orc_tinymt_single01(&rng[id]);
            int8_t* v = &a[(g0 + 1) * h + (g1 + 1)];
            if (cftp) {
                if ((double)rd < 0.5) {
                    if (*v == 3) *v = 12;
                } else if (*v == 12) {
                    *v = 3;
                }
            } else if ((double)rd < 0.8) {
                if (*v == 3)
                    *v = 12;
                else if (*v == 12)
                    *v = 3;
            }
        }
}

/* UpdateTiles, dominokernel.cl:22-31: each interior site of the other colour
 * takes its four edge bits from its four neighbours in the flipped array.
 * For a row of parity i%2, the neighbour towards j-1 sits at array column
 * j - (i+t+1)%2 and the one towards j+1 at j + (i+t)%2. */
static void domino_update(int8_t* dst, const int8_t* src, int n, int t) {
    const int h = n / 2;
    for (int i = 1; i <= n - 2; ++i)
        for (int j = 1; j <= h - 2; ++j) {
            const int up = src[(i - 1) * h + j], down = src[(i + 1) * h + j];
            const int west = src[i * h + j - (i + t + 1) % 2], east = src[i * h + j + (i + t) % 2];
            dst[i * h + j] = (int8_t)(((up & 2) >> 1) | ((down & 1) << 1) | ((west & 8) >> 1) | ((east & 4) << 1));
        }
}

static void domino_split(const int32_t* t, int n, int8_t* b, int8_t* w) {
    const int h = n / 2;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) ((i + j) % 2 == 0 ? b : w)[i * h + j / 2] = (int8_t)t[i * n + j];
}

static void domino_merge(int32_t* t, int n, const int8_t* b, const int8_t* w) {
    const int h = n / 2;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) t[i * n + j] = ((i + j) % 2 == 0 ? b : w)[i * h + j / 2];
}

static int domino_run(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k, int single_walk,
                      const uint32_t* params, int64_t nparams, int cftp) {
    if (n < 6 || n % 2) return ORC_EINVAL;
    const int h = n / 2;
    const int64_t items = (int64_t)(n - 2) * (h - 2);
    int8_t* b = (int8_t*)calloc((size_t)n * h, 1);
    int8_t* w = (int8_t*)calloc((size_t)n * h, 1);
    if (!b || !w) {
        free(b);
        free(w);
        return ORC_ENOMEM;
    }
    domino_split(t, n, b, w);
    int err = ORC_OK;
    for (int e = 0; e < k && err == ORC_OK; ++e) {
        mt_state m;
        mt_seed(&m, seeds[e]);
        /* single Walk: TinyMT seed = first mt19937 output (DominoTiler.cpp:31-32);
         * epoch Walk: TinyMT seed = seeds[k] itself (DominoTiler.cpp:81-82). */
        const uint32_t tseed = single_walk ? mt_next(&m) : (uint32_t)(uint64_t)seeds[e];
        orc_tinymt* rng = tmt_streams(items, tseed, params, nparams, &err);
        if (!rng) break;
        for (int64_t s = 0; s < steps[e]; ++s) {
            if (mt_next(&m) % 2u == 1u) {
                domino_rotate(b, n, rng, cftp);
                domino_update(w, b, n, 1);
            } else {
                domino_rotate(w, n, rng, cftp);
                domino_update(b, w, n, 0);
            }
        }
        free(rng);
    }
    if (err == ORC_OK) domino_merge(t, n, b, w);
    free(b);
    free(w);
    return err;
}

int orc_domino_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                    int cftp_kernel) {
    return domino_run(t, n, &steps, &seed, 1, 1, params, nparams, cftp_kernel);
}

int orc_domino_walk_epochs(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k,
                           const uint32_t* params, int64_t nparams, int cftp_kernel) {
    if (k < 0) return ORC_EINVAL;
    return domino_run(t, n, steps, seeds, k, 0, params, nparams, cftp_kernel);
}

/* ------------------------------------------------------------------------ */
/* Lozenge: src/Lozenge/LozengeTiler.cpp:18-88, lozengekernel.cl and        */
/* qlozengekernel.cl.  Vertex bits (LozengeTiler.h:11-17): 1 and 2 the two  */
/* upper edges, 4 and 8 the horizontal ones, 16 and 32 the lower ones; a    */
/* flippable vertex is 25 (1+8+16) or 38 (2+4+32).  Colour c of (i, j) is   */
/* ((j-i) mod 3); each colour is an N x N/3 array (column j/3).             */
/* ------------------------------------------------------------------------ */

/* RotateTiles, lozengekernel.cl:3-34 (uniform) and qlozengekernel.cl:5-32
 * (q-weighted).  Work item (i, j) owns stream j + (N/3) i. */
static void lozenge_rotate(void* arr, int isint, int n, orc_tinymt* rng, int qmode, double q, int qcmp) {
    const int m = n / 3;
    const float qf = (float)q;
    const float qinvf = 1.0f / qf;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) {
            const float rd = orc_tinymt_single01(&rng[(int64_t)j + (int64_t)m * i]);
            const int64_t at = (int64_t)i * m + j;
            const int v = isint ? ((int32_t*)arr)[at] : ((int8_t*)arr)[at];
            int nv = v;
            if (!qmode) {
                if ((double)rd < 0.4) {
                    if (v == 25) nv = 38;
                } else if ((double)rd < 0.8) {
                    if (v == 38) nv = 25;
                }
            } else if ((double)rd < 0.5) {
                const float x = rd / 0.5f; /* exact */
                const int ok = qcmp == ORC_QCMP_DOUBLE ? (q >= (double)x) : (qf >= x);
                if (v == 25 && ok) nv = 38;
            } else {
                const float x = (rd - 0.5f) * 0.5f; /* exact */
                const int ok = qcmp == ORC_QCMP_DOUBLE ? (1.0 / q >= (double)x) : (qinvf >= x);
                if (v == 38 && ok) nv = 25;
            }
            if (nv != v) {
                if (isint)
                    ((int32_t*)arr)[at] = nv;
                else
                    ((int8_t*)arr)[at] = (int8_t)nv;
            }
        }
}

/* UpdateTiles, lozengekernel.cl:36-54: after colour t flipped (array f), the
 * next colour (array a) refreshes bits {2,4,32} and the one after (array b)
 * bits {1,8,16} from f; the column shift of each neighbour depends on i mod 3. */
static void lozenge_update(const void* fv, void* av, void* bv, int isint, int n, int t) {
    const int m = n / 3;
#define LZ(arr, r, c) (isint ? ((const int32_t*)(arr))[(int64_t)(r)*m + (c)] : ((const int8_t*)(arr))[(int64_t)(r)*m + (c)])
    for (int i = 1; i <= n - 2; ++i) {
        const int r = i % 3;
        const int sa = r == (2 * t + 1) % 3; /* shift for the upper-right and lower-left reads */
        const int sw = r == (2 * t + 2) % 3;
        const int se = r == (2 * t) % 3;
        for (int j = 1; j <= m - 2; ++j) {
            const int a_old = LZ(av, i, j), b_old = LZ(bv, i, j);
            const int a_new = (a_old & ~38) + ((LZ(fv, i - 1, j + sa) & 16) >> 3) + ((LZ(fv, i, j - sw) & 8) >> 1) +
                              ((LZ(fv, i + 1, j) & 1) << 5);
            const int b_new = (b_old & ~25) + ((LZ(fv, i - 1, j) & 32) >> 5) + ((LZ(fv, i, j + se) & 4) << 1) +
                              ((LZ(fv, i + 1, j - sa) & 2) << 3);
            if (isint) {
                ((int32_t*)av)[(int64_t)i * m + j] = a_new;
                ((int32_t*)bv)[(int64_t)i * m + j] = b_new;
            } else {
                ((int8_t*)av)[(int64_t)i * m + j] = (int8_t)a_new;
                ((int8_t*)bv)[(int64_t)i * m + j] = (int8_t)b_new;
            }
        }
    }
#undef LZ
}

int orc_lozenge_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                     int qmode, double q, int qcmp) {
    if (n < 3 || n % 3) return ORC_EINVAL;
    const int m = n / 3;
    const int isint = qmode != 0; /* lozengekernel.cl stores char, qlozengekernel.cl int */
    const size_t es = isint ? 4 : 1;
    void* arr[3];
    for (int c = 0; c < 3; ++c) arr[c] = calloc((size_t)n * m, es);
    if (!arr[0] || !arr[1] || !arr[2]) {
        for (int c = 0; c < 3; ++c) free(arr[c]);
        return ORC_ENOMEM;
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const int c = ((j - i) % 3 + 3) % 3;
            const int64_t at = (int64_t)i * m + j / 3;
            if (isint)
                ((int32_t*)arr[c])[at] = t[(int64_t)i * n + j];
            else
                ((int8_t*)arr[c])[at] = (int8_t)t[(int64_t)i * n + j];
        }
    int err;
    orc_tinymt* rng = tmt_streams((int64_t)n * m, (uint32_t)(uint64_t)seed, params, nparams, &err);
    if (rng) {
        minstd g;
        minstd_seed(&g, seed);
        for (int64_t s = 0; s < steps; ++s) {
            const int r = uniform_int(&g, 2);
            lozenge_rotate(arr[r], isint, n, rng, qmode, q, qcmp);
            lozenge_update(arr[r], arr[(r + 1) % 3], arr[(r + 2) % 3], isint, n, r);
        }
        free(rng);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const int c = ((j - i) % 3 + 3) % 3;
                const int64_t at = (int64_t)i * m + j / 3;
                t[(int64_t)i * n + j] = isint ? ((int32_t*)arr[c])[at] : ((int8_t*)arr[c])[at];
            }
    }
    for (int c = 0; c < 3; ++c) free(arr[c]);
    return err;
}

/* ------------------------------------------------------------------------ */
/* Rectangle-triangle: src/RectTriangle/RectTriangleTiler.cpp:17-92 and     */
/* recttrianglekernel.cl.  A vertex holds its six face digits (hex digit k  */
/* = face k, RectTriangleTiler.h:16-21); colour of (i, j) is ((i-j) mod 3). */
/* ------------------------------------------------------------------------ */
static const float kRtDefaultWeights[16] = {0.0f, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};

static int hexd(int32_t x, int k) { return (int)(((uint32_t)x >> (4 * k)) & 0xfu); }

static float rt_weight(const float* w, int32_t x) {
    return w[hexd(x, 5)] * w[hexd(x, 4)] * w[hexd(x, 3)] * w[hexd(x, 2)] * w[hexd(x, 1)] * w[hexd(x, 0)];
}

/* flipTiles, recttrianglekernel.cl:25-118.  With probability 0.9 a site
 * proposes a move: a hexagon of the five-state cycle moves to the state that
 * the quarter of rd/0.9 selects (the member equal to itself standing in for
 * 0x122133); a site in one of six pair states toggles to its partner.  The
 * move is kept iff the face-weight ratio is >= the rescaled draw. */
static int32_t rt_propose(int32_t v, float rd, const float* w) {
    static const int32_t cyc[4] = {0xa7dd7a, 0xfc99cf, 0x8ebbe8, 0x331221};
    static const int32_t pairs[12] = {0x47d47a, 0xd22a33, 0xa74d74, 0x33a22d, 0x8eb558, 0x331eb1,
                                      0x855be8, 0x1be133, 0x6699cf, 0xcf1221, 0xfc9966, 0x1221fc};
    const float bs = 0.9f;
    if (!(rd < bs)) return v;
    rd = rd / bs;
    const int quarter = rd < 0.25f ? 0 : rd < 0.5f ? 1 : rd < 0.75f ? 2 : 3;
    float sc = (float)quarter * 0.25f;
    int32_t nv = v;
    if (v == 0x122133 || v == 0x331221 || v == 0x8ebbe8 || v == 0xfc99cf || v == 0xa7dd7a) {
        nv = cyc[quarter] == v ? 0x122133 : cyc[quarter];
    } else {
        for (int p = 0; p < 12; ++p)
            if (v == pairs[p]) {
                nv = pairs[p ^ 1];
                sc = 1.0f;
                break;
            }
    }
    const float ratio = rt_weight(w, nv) / rt_weight(w, v);
    const float x = sc == 1.0f ? rd : (rd - sc) * 4.0f;
    return ratio >= x ? nv : v;
}

static void rt_flip(int32_t* a, int n, orc_tinymt* rng, const float* w) {
    const int m = n / 3;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) {
            const float rd = orc_tinymt_single01(&rng[(int64_t)j + (int64_t)m * i]);
            int32_t* v = &a[(int64_t)i * m + j];
            *v = rt_propose(*v, rd, w);
        }
}

/* updateTiles1 / updateTiles2, recttrianglekernel.cl:120-146: each interior
 * site of the next (resp. the following) colour rebuilds its six face digits
 * from three flipped-colour neighbours; the column shift depends on i mod 3. */
static void rt_update(const int32_t* f, int32_t* a, int32_t* b, int n, int t) {
    const int m = n / 3;
#define F(r, c) f[(int64_t)(r)*m + (c)]
#define PUT(d, k) ((int32_t)(d) << (4 * (k)))
    for (int i = 1; i <= n - 2; ++i) {
        const int r = i % 3;
        const int s1 = r == t, s2 = r == (t + 1) % 3, s3 = r == (t + 2) % 3;
        for (int j = 1; j <= m - 2; ++j) {
            const int32_t up = F(i - 1, j), side = F(i, j + s1), low = F(i + 1, j - s2);
            a[(int64_t)i * m + j] = PUT(hexd(up, 1), 5) + PUT(hexd(up, 0), 4) + PUT(hexd(side, 5), 3) +
                                    PUT(hexd(low, 4), 2) + PUT(hexd(low, 3), 1) + PUT(hexd(side, 2), 0);
            const int32_t west = F(i, j - s3), upr = F(i - 1, j + s2), down = F(i + 1, j);
            b[(int64_t)i * m + j] = PUT(hexd(west, 3), 5) + PUT(hexd(upr, 2), 4) + PUT(hexd(upr, 1), 3) +
                                    PUT(hexd(west, 0), 2) + PUT(hexd(down, 5), 1) + PUT(hexd(down, 4), 0);
        }
    }
#undef F
#undef PUT
}

int orc_recttri_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                     const float* weights) {
    if (n < 3 || n % 3) return ORC_EINVAL;
    const float* w = weights ? weights : kRtDefaultWeights;
    const int m = n / 3;
    int32_t* arr[3];
    for (int c = 0; c < 3; ++c) arr[c] = (int32_t*)calloc((size_t)n * m, 4);
    if (!arr[0] || !arr[1] || !arr[2]) {
        for (int c = 0; c < 3; ++c) free(arr[c]);
        return ORC_ENOMEM;
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) arr[((i - j) % 3 + 3) % 3][(int64_t)i * m + j / 3] = t[(int64_t)i * n + j];
    int err;
    orc_tinymt* rng = tmt_streams((int64_t)n * m, (uint32_t)(uint64_t)seed, params, nparams, &err);
    if (rng) {
        minstd g;
        minstd_seed(&g, seed);
        for (int64_t s = 0; s < steps; ++s) {
            const int r = uniform_int(&g, 2);
            rt_flip(arr[r], n, rng, w);
            rt_update(arr[r], arr[(r + 1) % 3], arr[(r + 2) % 3], n, r);
        }
        free(rng);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) t[(int64_t)i * n + j] = arr[((i - j) % 3 + 3) % 3][(int64_t)i * m + j / 3];
    }
    for (int c = 0; c < 3; ++c) free(arr[c]);
    return err;
}

/* Triangular-lattice dimers: not yet restated. */
int orc_tridimer_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams) {
    (void)t;
    (void)n;
    (void)steps;
    (void)seed;
    (void)params;
    (void)nparams;
    return ORC_EINVAL;
}
