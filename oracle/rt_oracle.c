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

#include <math.h>
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
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as  */
/* easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies by      */
/* 0xD2511F53 / 0xCD9E8D57, key bumped by the Weyl constants 0x9E3779B9 /   */
/* 0xBB67AE85 between rounds.  The fast mode's counter-based generator; it  */
/* has no counterpart in the reference.                                     */
/* ------------------------------------------------------------------------ */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0, out[1] = c1, out[2] = c2, out[3] = c3;
}

/* Where a Rotate's draws come from.  Bit-exact mode: the reference's TinyMT
 * stream of work item c + cols * r.  Fast mode: work item (r, c) acts on site
 * (i, j) = (r + roff, c + coff) of its colour array (`width` sites per row);
 * the site belongs to quad u = i * ceil(width / 4) + j / 4 -- the 32-bit word
 * of four int8 sites that holds it -- and takes output word j mod 4 of
 * Philox4x32-10(counter = (u, step lo, step hi, chain), key), where `step`
 * counts the drawing steps of the epoch from 0.  Either way the draw is
 * k * 2^-23 with a 23-bit k (the top bits of the 32-bit word). */
typedef struct {
    int fast;
    orc_tinymt* tmt;
    int64_t cols;
    int64_t roff, coff, width;
    uint32_t key[2], chain;
    uint64_t step;
    int64_t cached_u; /* quad whose words are in w[] (-1: none) */
    uint32_t w[4];
} orc_draws;

static float orc_draw(orc_draws* d, int64_t r, int64_t c) {
    if (!d->fast) return orc_tinymt_single01(&d->tmt[c + d->cols * r]);
    const int64_t i = r + d->roff, j = c + d->coff;
    const int64_t u = i * ((d->width + 3) / 4) + j / 4;
    if (u != d->cached_u) {
        const uint32_t ctr[4] = {(uint32_t)u, (uint32_t)d->step, (uint32_t)(d->step >> 32), d->chain};
        orc_philox4x32_10(ctr, d->key, d->w);
        d->cached_u = u;
    }
    return (float)(d->w[j & 3] >> 9) * (1.0f / 8388608.0f);
}

/* Bit-plane mode (no reference counterpart): one random bit per site.  Site
 * (i, j) of a colour array `width` sites wide lies in 32-bit word j / 32 of
 * its row, and words come in fours: quad q = j / 128 of band row g = i -
 * roff takes Philox4x32-10(counter = (g * ceil(ceil(width / 32) / 4) + q,
 * step lo, step hi, chain), key) and word (j / 32) mod 4 of the output; the
 * site's bit is bit j mod 32 of that word.  `second` selects the second bit
 * of the domino toggle rule (counter word 0 with its top bit set). */
static int plane_bit(const orc_draws* d, int64_t i, int64_t j, int second) {
    const int64_t ww = (d->width + 31) / 32, qpr = (ww + 3) / 4;
    const uint32_t c0 = (uint32_t)((i - d->roff) * qpr + (j / 32) / 4) | (second ? 0x80000000u : 0u);
    const uint32_t ctr[4] = {c0, (uint32_t)d->step, (uint32_t)(d->step >> 32), d->chain};
    uint32_t out[4];
    orc_philox4x32_10(ctr, d->key, out);
    return (int)((out[(j / 32) & 3] >> (j & 31)) & 1u);
}

/* Starts an epoch: TinyMT streams seeded with `seed` (bit-exact mode) or the
 * Philox key `seed` (fast mode).  Work item (r, c) of the Rotate range (cols
 * items per row) acts on site (r + roff, c + coff) of a colour array `width`
 * sites wide. */
static int draws_begin(orc_draws* d, int fast, int64_t items, int64_t cols, int64_t roff, int64_t coff,
                       int64_t width, uint64_t seed, uint32_t chain, const uint32_t* params, int64_t nparams) {
    int err = ORC_OK;
    memset(d, 0, sizeof *d);
    d->fast = fast;
    d->cols = cols;
    d->roff = roff;
    d->coff = coff;
    d->width = width;
    d->chain = chain;
    d->cached_u = -1;
    if (fast) {
        d->key[0] = (uint32_t)seed;
        d->key[1] = (uint32_t)(seed >> 32);
    } else {
        d->tmt = tmt_streams(items, (uint32_t)seed, params, nparams, &err);
    }
    return err;
}
/* After every Rotate: the next step's counters. */
static void draws_next(orc_draws* d) {
    d->step++;
    d->cached_u = -1;
}
static void draws_end(orc_draws* d) {
    free(d->tmt);
    d->tmt = NULL;
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
/* Periodic domino weights (no reference counterpart): NULL = uniform. */
typedef struct {
    int period;
    const double* wh; /* horizontal domino on squares (r, c), (r, c+1): wh[(r mod P) P + c mod P] */
    const double* wv; /* vertical domino on squares (r, c), (r+1, c) */
} orc_weights;

static double weight_at(const double* w, int P, int r, int c) { return w[(((r % P) + P) % P) * P + (((c % P) + P) % P)]; }

/* Heat-bath probability of state 12 (two vertical dominoes) at vertex (i, j):
 * w12 / (w3 + w12), w3 the two horizontal dominoes' weights (squares
 * (i-1, j-1)-(i-1, j) and (i, j-1)-(i, j)), w12 the two vertical ones'
 * ((i-1, j-1)-(i, j-1) and (i-1, j)-(i, j)). */
static double weighted_p12(const orc_weights* w, int i, int j) {
    const int P = w->period;
    const double w3 = weight_at(w->wh, P, i - 1, j - 1) * weight_at(w->wh, P, i, j - 1);
    const double w12 = weight_at(w->wv, P, i - 1, j - 1) * weight_at(w->wv, P, i - 1, j);
    return w12 / (w3 + w12);
}

static void domino_rotate(int8_t* a, int n, orc_draws* rng, int cftp, const orc_weights* wts, int black) {
    const int h = n / 2, gw = h - 2;
    for (int g0 = 0; g0 < n - 2; ++g0)
        for (int g1 = 0; g1 < gw; ++g1) {
            const float rd = orc_draw(rng, g0, g1);
            int8_t* v = &a[(g0 + 1) * h + (g1 + 1)];
            if (cftp) {
                /* array column c of the black / white array is vertex column 2c + parity */
                const int i = g0 + 1, j = 2 * (g1 + 1) + (black ? (i & 1) : 1 - (i & 1));
                const double p = wts ? weighted_p12(wts, i, j) : 0.5;
                if ((double)rd < p) {
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

/* Bit-plane mode Rotate (no reference counterpart): heat bath -- a rotatable
 * site (3 or 12) becomes 12 where its bit is 1, else 3; toggle -- 3 <-> 12
 * where either of its two bits is 1. */
static void domino_rotate_planes(int8_t* a, int n, const orc_draws* rng, int heat_bath) {
    const int h = n / 2;
    for (int i = 1; i <= n - 2; ++i)
        for (int j = 1; j <= h - 2; ++j) {
            int8_t* v = &a[i * h + j];
            if (*v != 3 && *v != 12) continue;
            if (heat_bath)
                *v = plane_bit(rng, i, j, 0) ? 12 : 3;
            else if (plane_bit(rng, i, j, 0) | plane_bit(rng, i, j, 1))
                *v = (int8_t)(*v ^ 15);
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
                      const uint32_t* params, int64_t nparams, int cftp, int fast, uint32_t chain,
                      const orc_weights* wts) {
    /* fast == 2: bit-plane mode (Philox bits, same colour cycle as fast mode) */
    const int planes = fast == 2;
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
         * epoch Walk: TinyMT seed = seeds[k] itself (DominoTiler.cpp:81-82).
         * Fast mode: the Philox key is the seed and the colours alternate,
         * black ((i+j) even) first. */
        const uint64_t tseed = fast ? (uint64_t)seeds[e] : single_walk ? mt_next(&m) : (uint32_t)(uint64_t)seeds[e];
        orc_draws rng;
        err = draws_begin(&rng, fast, items, h - 2, 1, 1, h, tseed, chain, params, nparams);
        if (err != ORC_OK) break;
        for (int64_t s = 0; s < steps[e]; ++s) {
            const int black = fast ? (s & 1) == 0 : mt_next(&m) % 2u == 1u;
            if (black) {
                if (planes)
                    domino_rotate_planes(b, n, &rng, cftp);
                else
                    domino_rotate(b, n, &rng, cftp, wts, 1);
                domino_update(w, b, n, 1);
            } else {
                if (planes)
                    domino_rotate_planes(w, n, &rng, cftp);
                else
                    domino_rotate(w, n, &rng, cftp, wts, 0);
                domino_update(b, w, n, 0);
            }
            draws_next(&rng);
        }
        draws_end(&rng);
    }
    if (err == ORC_OK) domino_merge(t, n, b, w);
    free(b);
    free(w);
    return err;
}

int orc_domino_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                    int cftp_kernel) {
    return domino_run(t, n, &steps, &seed, 1, 1, params, nparams, cftp_kernel, 0, 0, NULL);
}

int orc_domino_walk_epochs(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k,
                           const uint32_t* params, int64_t nparams, int cftp_kernel) {
    if (k < 0) return ORC_EINVAL;
    return domino_run(t, n, steps, seeds, k, 0, params, nparams, cftp_kernel, 0, 0, NULL);
}

int orc_domino_walk_fast(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain,
                         int cftp_kernel) {
    if (k < 0) return ORC_EINVAL;
    return domino_run(t, n, steps, keys, k, 0, NULL, 0, cftp_kernel, 1, chain, NULL);
}

int orc_domino_walk_weighted(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k, int single_walk,
                             int fast, uint32_t chain, const uint32_t* params, int64_t nparams, int period,
                             const double* wh, const double* wv) {
    if (k < 0 || (period != 1 && period != 2 && period != 4) || !wh || !wv) return ORC_EINVAL;
    const orc_weights w = {period, wh, wv};
    return domino_run(t, n, steps, seeds, k, single_walk, params, nparams, 1, fast ? 1 : 0, chain, &w);
}

int orc_domino_walk_planes(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain,
                           int heat_bath) {
    if (k < 0) return ORC_EINVAL;
    return domino_run(t, n, steps, keys, k, 0, NULL, 0, heat_bath, 2, chain, NULL);
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
/* Periodic lozenge weights (no reference counterpart): a lozenge weighs the
 * table entry of the lattice edge it covers, named by its lower end (i, j):
 * w[0] the edge to (i, j+1), w[1] to (i-1, j+1), w[2] to (i-1, j). */
typedef struct {
    int period;
    const double* w[3];
} orc_lweights;

/* Probability of state 38 (the cube) at vertex (i, j): W38 / (W25 + W38). */
static double lozenge_p38(const orc_lweights* lw, int i, int j) {
    const int P = lw->period;
    const double w25 = weight_at(lw->w[2], P, i, j) * weight_at(lw->w[0], P, i, j) * weight_at(lw->w[1], P, i + 1, j - 1);
    const double w38 = weight_at(lw->w[1], P, i, j) * weight_at(lw->w[0], P, i, j - 1) * weight_at(lw->w[2], P, i + 1, j);
    return w38 / (w25 + w38);
}

static void lozenge_rotate(void* arr, int isint, int n, orc_draws* rng, int qmode, double q, int qcmp,
                           const orc_lweights* lw, int colour) {
    const int m = n / 3;
    const float qf = (float)q;
    const float qinvf = 1.0f / qf;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) {
            const float rd = orc_draw(rng, i, j);
            const int64_t at = (int64_t)i * m + j;
            const int v = isint ? ((int32_t*)arr)[at] : ((int8_t*)arr)[at];
            int nv = v;
            if (lw) {
                /* array column j of this colour is vertex column 3j + (colour + i) mod 3 */
                const double add = 0.8 * lozenge_p38(lw, i, 3 * j + (colour + i) % 3);
                if ((double)rd < add) {
                    if (v == 25) nv = 38;
                } else if ((double)rd < 0.8) {
                    if (v == 38) nv = 25;
                }
            } else if (qmode == 2) {
                /* volume weight q in the int8 fast rule of the batched chains: add below 0.4 q */
                if ((double)rd < 0.4 * q) {
                    if (v == 25) nv = 38;
                } else if ((double)rd >= 0.4 && (double)rd < 0.8) {
                    if (v == 38) nv = 25;
                }
            } else if (!qmode) {
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
/* Bit-plane mode Rotate (no reference counterpart): heat bath -- 25 -> 38
 * (add a cube) where the site's bit is 1, 38 -> 25 where it is 0. */
static void lozenge_rotate_planes(int8_t* a, int n, const orc_draws* rng) {
    const int m = n / 3;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) {
            int8_t* v = &a[(int64_t)i * m + j];
            if (*v == 25 && plane_bit(rng, i, j, 0)) *v = 38;
            else if (*v == 38 && !plane_bit(rng, i, j, 0)) *v = 25;
        }
}

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

/* Epochs as the domino epoch Walk composes them (DominoTiler.cpp:58-107):
 * epoch e restarts the colour engine and the draws from seeds[e].  The
 * reference's single Walk (LozengeTiler.cpp:18-88) is the one-epoch case. */
static int lozenge_run(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k, const uint32_t* params,
                       int64_t nparams, int qmode, double q, int qcmp, int fast, uint32_t chain,
                       const orc_lweights* lw) {
    if (n < 3 || n % 3 || k < 0) return ORC_EINVAL;
    const int m = n / 3;
    const int isint = qmode == 1; /* lozengekernel.cl stores char, qlozengekernel.cl int */
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
    int err = ORC_OK;
    for (int e = 0; e < k && err == ORC_OK; ++e) {
        orc_draws rng;
        err = draws_begin(&rng, fast, (int64_t)n * m, m, 0, 0, m,
                          fast ? (uint64_t)seeds[e] : (uint32_t)(uint64_t)seeds[e], chain, params, nparams);
        if (err != ORC_OK) break;
        minstd g;
        minstd_seed(&g, seeds[e]);
        for (int64_t s = 0; s < steps[e]; ++s) {
            const int r = fast ? (int)(s % 3) : uniform_int(&g, 2);
            if (fast == 2)
                lozenge_rotate_planes((int8_t*)arr[r], n, &rng);
            else
                lozenge_rotate(arr[r], isint, n, &rng, qmode, q, qcmp, lw, r);
            lozenge_update(arr[r], arr[(r + 1) % 3], arr[(r + 2) % 3], isint, n, r);
            draws_next(&rng);
        }
        draws_end(&rng);
    }
    if (err == ORC_OK)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const int c = ((j - i) % 3 + 3) % 3;
                const int64_t at = (int64_t)i * m + j / 3;
                t[(int64_t)i * n + j] = isint ? ((int32_t*)arr[c])[at] : ((int8_t*)arr[c])[at];
            }
    for (int c = 0; c < 3; ++c) free(arr[c]);
    return err;
}

/* The first step count after which the q-weighted walk (qlozengekernel.cl,
 * TinyMT32J streams, seed) differs between the float32 and the double
 * comparison, or 0 when it does not within max_steps.  Both walks agree up to
 * the first draw that a site can accept in one comparison and not in the
 * other, so one walk in the double comparison finds it.  Used to pick fixture
 * step counts that tell the two comparisons apart. */
int64_t orc_lozenge_q_divergence(const int32_t* t, int n, int64_t seed, int64_t max_steps, double q) {
    if (n < 3 || n % 3) return -1;
    const int m = n / 3;
    const float qf = (float)q, qinvf = 1.0f / qf;
    int32_t* arr[3];
    for (int c = 0; c < 3; ++c) arr[c] = calloc((size_t)n * m, 4);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) arr[((j - i) % 3 + 3) % 3][(int64_t)i * m + j / 3] = t[(int64_t)i * n + j];
    orc_draws rng;
    int64_t found = 0;
    if (draws_begin(&rng, 0, (int64_t)n * m, m, 0, 0, m, (uint32_t)(uint64_t)seed, 0, NULL, 0) != ORC_OK) found = -1;
    minstd g;
    minstd_seed(&g, seed);
    for (int64_t s = 0; s < max_steps && found == 0; ++s) {
        const int r = uniform_int(&g, 2);
        /* the Rotate of qlozengekernel.cl:18-29 in the double comparison, watching the float32 one */
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < m; ++j) {
                const float rd = orc_draw(&rng, i, j);
                int32_t* v = &arr[r][(int64_t)i * m + j];
                if (rd < 0.5f) {
                    const float x = rd / 0.5f;
                    const int okd = q >= (double)x, okf = qf >= x;
                    if (*v == 25 && okd != okf && found == 0) found = s + 1;
                    if (*v == 25 && okd) *v = 38;
                } else {
                    const float x = (rd - 0.5f) * 0.5f;
                    const int okd = 1.0 / q >= (double)x, okf = qinvf >= x;
                    if (*v == 38 && okd != okf && found == 0) found = s + 1;
                    if (*v == 38 && okd) *v = 25;
                }
            }
        lozenge_update(arr[r], arr[(r + 1) % 3], arr[(r + 2) % 3], 1, n, r);
        draws_next(&rng);
    }
    if (found >= 0) draws_end(&rng);
    for (int c = 0; c < 3; ++c) free(arr[c]);
    return found;
}

int orc_lozenge_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                     int qmode, double q, int qcmp) {
    return lozenge_run(t, n, &steps, &seed, 1, params, nparams, qmode, q, qcmp, 0, 0, NULL);
}

int orc_lozenge_walk_epochs(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k,
                            const uint32_t* params, int64_t nparams, int qmode, double q, int qcmp) {
    return lozenge_run(t, n, steps, seeds, k, params, nparams, qmode, q, qcmp, 0, 0, NULL);
}

int orc_lozenge_walk_fast(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain,
                          int qmode, double q, int qcmp) {
    return lozenge_run(t, n, steps, keys, k, NULL, 0, qmode, q, qcmp, 1, chain, NULL);
}

int orc_lozenge_walk_planes(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain) {
    return lozenge_run(t, n, steps, keys, k, NULL, 0, 0, 1.0, 0, 2, chain, NULL);
}

int orc_lozenge_walk_weighted(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k, int fast,
                              uint32_t chain, const uint32_t* params, int64_t nparams, int period, const double* w0,
                              const double* w1, const double* w2) {
    if (k < 0 || (period != 1 && period != 2 && period != 4) || !w0 || !w1 || !w2) return ORC_EINVAL;
    const orc_lweights lw = {period, {w0, w1, w2}};
    return lozenge_run(t, n, steps, seeds, k, params, nparams, 0, 1.0, 0, fast ? 1 : 0, chain, &lw);
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

static void rt_flip(int32_t* a, int n, orc_draws* rng, const float* w) {
    const int m = n / 3;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) {
            const float rd = orc_draw(rng, i, j);
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

static int recttri_run(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                       const float* weights, int fast, uint32_t chain) {
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
    orc_draws rng;
    int err = draws_begin(&rng, fast, (int64_t)n * m, m, 0, 0, m, fast ? (uint64_t)seed : (uint32_t)(uint64_t)seed,
                          chain, params, nparams);
    if (err == ORC_OK) {
        minstd g;
        minstd_seed(&g, seed);
        for (int64_t s = 0; s < steps; ++s) {
            const int r = fast ? (int)(s % 3) : uniform_int(&g, 2);
            rt_flip(arr[r], n, &rng, w);
            rt_update(arr[r], arr[(r + 1) % 3], arr[(r + 2) % 3], n, r);
            draws_next(&rng);
        }
        draws_end(&rng);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) t[(int64_t)i * n + j] = arr[((i - j) % 3 + 3) % 3][(int64_t)i * m + j / 3];
    }
    for (int c = 0; c < 3; ++c) free(arr[c]);
    return err;
}

int orc_recttri_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                     const float* weights) {
    return recttri_run(t, n, steps, seed, params, nparams, weights, 0, 0);
}

int orc_recttri_walk_fast(int32_t* t, int n, int64_t steps, int64_t key, uint32_t chain, const float* weights) {
    return recttri_run(t, n, steps, key, NULL, 0, weights, 1, chain);
}

/* ------------------------------------------------------------------------ */
/* Triangular-lattice dimers (bibone): src/TriangleDimer/TriangleDimerTiler */
/* .cpp:86-483 and triangledimerkernel.cl.  Eight M x M int arrays (M =     */
/* N/2): lozenge states H, L, R; triangle states U, D; butterfly states     */
/* BH, BL, BR.  Each step flips one family (lozenge / triangle / butterfly) */
/* of one orientation and class, then recomputes the dependent arrays by a  */
/* fixed sequence of kernels; every kernel below is one NDRange (M, M),     */
/* restated as a serial loop (each is race-free).                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int m;
    int32_t *H, *L, *R, *U, *D, *BH, *BL, *BR;
} td_state;

#define TD(a, i, j) ((a)[(int64_t)(i) * st->m + (j)])
#define TD_INTERIOR(i, j) ((i) >= 1 && (i) <= st->m - 2 && (j) >= 1 && (j) <= st->m - 2)

static int dg(int32_t x, int k) { return (int)(((uint32_t)x >> (2 * k)) & 3u); } /* base-4 digit */
static int cycle_up(int d) { return d == 0 ? 0 : d % 3 + 1; }          /* 1->2, 2->3, 3->1 */
static int cycle_down(int d) { return d == 0 ? 0 : (d + 1) % 3 + 1; }  /* 1->3, 2->1, 3->2 */
static int32_t bf_pack(int t1, int t4, int t16, int t64, int c) { return t1 + 4 * t4 + 16 * t16 + 64 * t64 + 256 * c; }

/* RotateLozenges (triangledimerkernel.cl:4-22): every item draws; sites of
 * orientation t and checkerboard class c toggle 5 <-> 10 when rd < .5. */
static void td_rotate_lozenges(td_state* st, int32_t* A, int t, int c, orc_draws* rng) {
    const int m = st->m;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            const float rd = orc_draw(rng, i, j);
            const int cls = ((1 - (t & 1)) * i + ((1 + t) / 2) * j) % 2;
            if ((double)rd < 0.5 && cls == c) {
                int32_t* v = &TD(A, i, j);
                if (*v == 5) *v = 10;
                else if (*v == 10) *v = 5;
            }
        }
}

/* UpdateLozengesFlipped (:24-33): sites of the other class of the same
 * orientation, from their four neighbours of the flipped class. */
static void td_lozenges_flipped(td_state* st, int32_t* A, int t, int c) {
    const int dj = t & 1, di = (2 - t) / 2;
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            const int cls = ((1 - (t & 1)) * i + ((1 + t) / 2) * j) % 2;
            if (cls == c) continue;
            TD(A, i, j) = ((TD(A, i - 1, j + dj) >> 2) & 1) | (((TD(A, i - di, j + 1) >> 3) & 1) << 1) |
                          ((TD(A, i + 1, j - dj) & 1) << 2) | (((TD(A, i + di, j - 1) >> 1) & 1) << 3);
        }
}

/* UpdateLozenges0/1/2 (:35-78): the two other orientations take the bits they
 * share with the flipped one. */
static void td_lozenges_other(td_state* st, int t) {
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            if (t == 0) {
                const int32_t* f = st->H;
                TD(st->L, i, j) = (TD(st->L, i, j) & ~10) | ((TD(f, i + 1, j) & 1) << 1) | ((TD(f, i + 1, j - 1) & 1) << 3);
                TD(st->R, i, j) = (TD(st->R, i, j) & ~10) | (TD(f, i + 1, j) & 2) | (TD(f, i, j) & 8);
            } else if (t == 1) {
                const int32_t* f = st->L;
                TD(st->R, i, j) = (TD(st->R, i, j) & ~5) | (TD(f, i, j) & 1) | ((TD(f, i + 1, j) & 1) << 2);
                TD(st->H, i, j) = (TD(st->H, i, j) & ~5) | ((TD(f, i - 1, j) & 2) >> 1) | ((TD(f, i, j) & 2) << 1);
            } else {
                const int32_t* f = st->R;
                TD(st->H, i, j) = (TD(st->H, i, j) & ~10) | (TD(f, i - 1, j) & 2) | ((TD(f, i, j - 1) & 2) << 2);
                TD(st->L, i, j) = (TD(st->L, i, j) & ~5) | (TD(f, i, j) & 1) | (TD(f, i, j - 1) & 4);
            }
        }
}

/* UpdateTriangleUFromLozenges (:96-116). */
static void td_up_from_lozenges(td_state* st) {
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            const int32_t l0 = TD(st->L, i, j), l1 = TD(st->L, i, j + 1), h0 = TD(st->H, i, j), h1 = TD(st->H, i + 1, j);
            const int a = ((l0 & 1) ? 1 : 0) + ((h0 & 8) ? 2 : 0) + ((h1 & 1) ? 3 : 0);
            const int b = ((l1 & 1) ? 1 : 0) + ((h1 & 2) ? 2 : 0) + ((l1 & 2) ? 3 : 0);
            const int c = ((l1 & 4) ? 1 : 0) + ((h1 & 8) ? 2 : 0) + ((h1 & 4) ? 3 : 0);
            TD(st->U, i, j) = a + 4 * b + 16 * c;
        }
}

/* UpdateButterflys{H,L,R}FromLozenge (:118-189). */
static void td_butterfly_from_lozenges(td_state* st, int which) {
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            int t1, t4, t16, t64, c;
            if (which == 0) {
                const int32_t h = TD(st->H, i, j), ru = TD(st->R, i - 1, j), lu = TD(st->L, i - 1, j + 1);
                const int32_t r = TD(st->R, i, j), l = TD(st->L, i, j);
                c = (lu >> 2) & 1;
                t1 = ((ru >> 3) & 1) + 2 * (ru & 1) + 3 * (h & 1);
                t4 = (lu & 1) + (lu & 2) + 3 * ((h >> 1) & 1);
                t16 = ((r >> 1) & 1) + ((r >> 1) & 2) + 3 * ((h >> 2) & 1);
                t64 = ((l >> 2) & 1) + ((l >> 2) & 2) + 3 * ((h >> 3) & 1);
                TD(st->BH, i, j) = bf_pack(t1, t4, t16, t64, c);
            } else if (which == 1) {
                const int32_t l = TD(st->L, i, j), h = TD(st->H, i, j), r = TD(st->R, i, j);
                const int32_t hd = TD(st->H, i + 1, j - 1), rw = TD(st->R, i, j - 1);
                c = (r >> 3) & 1;
                t1 = (h & 1) + (h & 2) + 3 * (l & 1);
                t4 = ((r >> 1) & 1) + ((r >> 1) & 2) + 3 * ((l >> 1) & 1);
                t16 = ((hd >> 2) & 1) + ((hd >> 2) & 2) + 3 * ((l >> 2) & 1);
                t64 = ((rw >> 3) & 1) + 2 * (rw & 1) + 3 * ((l >> 3) & 1);
                TD(st->BL, i, j) = bf_pack(t1, t4, t16, t64, c);
            } else {
                const int32_t r = TD(st->R, i, j), h = TD(st->H, i, j), le = TD(st->L, i, j + 1);
                const int32_t hd = TD(st->H, i + 1, j), l = TD(st->L, i, j);
                c = (le >> 3) & 1;
                t1 = (h & 1) + (h & 2) + 3 * (r & 1);
                t4 = (le & 1) + (le & 2) + 3 * ((r >> 1) & 1);
                t16 = ((hd >> 2) & 1) + ((hd >> 2) & 2) + 3 * ((r >> 2) & 1);
                t64 = ((l >> 2) & 1) + ((l >> 2) & 2) + 3 * ((r >> 3) & 1);
                TD(st->BR, i, j) = bf_pack(t1, t4, t16, t64, c);
            }
        }
}

/* RotateTriangles (:191-211): class ((j-i) mod 3) == c toggles 45 <-> 54. */
static void td_rotate_triangles(td_state* st, int32_t* A, int c, orc_draws* rng) {
    const int m = st->m;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            const float rd = orc_draw(rng, i, j);
            if ((double)rd < 0.5 && ((j - i) % 3 + 3) % 3 == c) {
                int32_t* v = &TD(A, i, j);
                if (*v == 45) *v = 54;
                else if (*v == 54) *v = 45;
            }
        }
}

/* UpdateTrianglesFlipped0/1 (:213-253): same-kind triangles of the other two
 * classes, one base-4 digit from each of three flipped-class neighbours. */
static void td_triangles_flipped(td_state* st, int32_t* A, int up, int c) {
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            const int cls = ((j - i) % 3 + 3) % 3;
            if (cls == c) continue;
            const int p = cls == (c + 1) % 3;
            int32_t v;
            if (up)
                v = p ? dg(TD(A, i, j - 1), 1) + 4 * dg(TD(A, i - 1, j + 1), 2) + 16 * dg(TD(A, i + 1, j), 0)
                      : dg(TD(A, i - 1, j), 2) + 4 * dg(TD(A, i, j + 1), 0) + 16 * dg(TD(A, i + 1, j - 1), 1);
            else
                v = p ? dg(TD(A, i, j - 1), 1) + 4 * dg(TD(A, i + 1, j), 2) + 16 * dg(TD(A, i - 1, j + 1), 0)
                      : dg(TD(A, i + 1, j - 1), 2) + 4 * dg(TD(A, i, j + 1), 0) + 16 * dg(TD(A, i - 1, j), 1);
            TD(A, i, j) = v;
        }
}

/* UpdateTriangles (:255-275): down from up (t=0) or up from down (t=1). */
static int td_tri_digit(int32_t v) {
    return ((v & 48) == 16 ? 1 : 0) + ((v & 3) == 3 ? 2 : 0) + ((v & 12) == 8 ? 3 : 0);
}
static void td_triangles_other(td_state* st, const int32_t* A, int32_t* B, int t) {
    const int p = t == 0 ? -1 : 1;
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j)
            TD(B, i, j) = td_tri_digit(TD(A, i, j - 1 + t)) + 4 * td_tri_digit(TD(A, i, j + t)) +
                          16 * td_tri_digit(TD(A, i + p, j));
}

/* UpdateLozenge{H,L,R}FromTriangles (:277-329). */
static void td_lozenges_from_triangles(td_state* st) {
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            const int32_t d = TD(st->D, i, j);
            const int32_t uh = TD(st->U, i - 1, j), ul = TD(st->U, i, j - 1), ur = TD(st->U, i, j);
            TD(st->H, i, j) = ((d & 48) == 32) + 2 * ((d & 48) == 48) + 4 * ((uh & 48) == 48) + 8 * ((uh & 48) == 32);
            TD(st->L, i, j) = ((ul & 12) == 4) + 2 * ((ul & 12) == 12) + 4 * ((d & 3) == 1) + 8 * ((d & 3) == 2);
            TD(st->R, i, j) = ((ur & 3) == 1) + 2 * ((d & 12) == 12) + 4 * ((d & 12) == 4) + 8 * ((ur & 3) == 2);
        }
}

/* RotateButterflys (:331-353): slice (b1 i + b2 j) mod 3 == p1; within it the
 * sites of parity p2 toggle 170 <-> 85 when rd < .5. */
static void td_rotate_butterflies(td_state* st, int32_t* A, int t, int p1, int p2, orc_draws* rng) {
    const int m = st->m;
    const int b1 = 1 - (t & 1), b2 = (1 + t) / 2, b3 = t & 1;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            const float rd = orc_draw(rng, i, j);
            if ((double)rd < 0.5 && (b1 * i + b2 * j) % 3 == p1 && ((b1 * j + b3 * i) & 1) == p2) {
                int32_t* v = &TD(A, i, j);
                if (*v == 170) *v = 85;
                else if (*v == 85) *v = 170;
            }
        }
}

/* The three-pass butterfly update after a butterfly flip
 * (UpdateButterflysFlipped{H,L,R}{1,21,22,23}, :356-652).  For orientation
 * t the slice index and the positions of the neighbours differ; `nb` gives
 * the neighbour cells of each pass. */
static int td_slice(int t, int i, int j) { return t == 0 ? i % 3 : t == 1 ? j % 3 : (i + j) % 3; }
static int td_par(int t, int i, int j) { return t == 1 ? (i & 1) : (j & 1); }

static void td_butterfly_same_slice(td_state* st, int32_t* B, int t, int p1, int p2) {
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            if (td_slice(t, i, j) != p1 || td_par(t, i, j) == p2) continue;
            const int c = (TD(B, i, j) >> 8) & 1;
            int t1, t4, t16, t64;
            if (t == 2) {
                const int32_t lo = TD(B, i + 1, j - 1), hi = TD(B, i - 1, j + 1);
                t1 = cycle_down(dg(hi, 3));
                t4 = cycle_up(dg(hi, 2));
                t16 = cycle_down(dg(lo, 1));
                t64 = cycle_up(dg(lo, 0));
            } else {
                const int32_t a = t == 0 ? TD(B, i, j - 1) : TD(B, i - 1, j);
                const int32_t b = t == 0 ? TD(B, i, j + 1) : TD(B, i + 1, j);
                t1 = cycle_up(dg(a, 1));
                t4 = cycle_down(dg(b, 0));
                t16 = cycle_up(dg(b, 3));
                t64 = cycle_down(dg(a, 2));
            }
            TD(B, i, j) = bf_pack(t1, t4, t16, t64, c);
        }
}

/* Pass 21 (first half of the adjacent slice) for H and L; R's first pass
 * touches the slice p1+2 as well.  H: slice p1+1, neighbours above;
 * L: slice p1+2, neighbours to the right; R: slice p1+2. */
static void td_butterfly_pass21(td_state* st, int32_t* B, int t, int p1) {
    const int want = t == 0 ? (p1 + 1) % 3 : (p1 + 2) % 3;
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            if (td_slice(t, i, j) != want) continue;
            const int32_t f = TD(B, i, j);
            int t1, t4, t16, t64, c;
            if (t == 2) {
                const int32_t e = TD(B, i, j + 1), s = TD(B, i + 1, j);
                c = dg(s, 0) == 1;
                t1 = dg(f, 0);
                t4 = dg(f, 1) == 2 ? 2 : (dg(e, 0) == 3) + 3 * (dg(e, 3) == 3);
                t16 = dg(f, 2) == 1 ? 1 : 3 * (dg(s, 0) == 3) + 2 * (dg(s, 3) == 3);
                t64 = dg(f, 3);
            } else {
                const int32_t a = t == 0 ? TD(B, i - 1, j) : TD(B, i - 1, j + 1);
                const int32_t b = t == 0 ? TD(B, i - 1, j + 1) : TD(B, i, j + 1);
                c = dg(a, 2) == 2;
                t1 = dg(f, 0) == 2 ? 2 : (dg(a, 3) == 3) + 3 * (dg(a, 2) == 3);
                t4 = dg(f, 1) == 1 ? 1 : 3 * (dg(b, 3) == 3) + 2 * (dg(b, 2) == 3);
                t16 = dg(f, 2);
                t64 = dg(f, 3);
            }
            TD(B, i, j) = bf_pack(t1, t4, t16, t64, c);
        }
}

/* Pass 22: the other adjacent slice (H: p1+2, L and R: p1+1). */
static void td_butterfly_pass22(td_state* st, int32_t* B, int t, int p1) {
    const int want = t == 0 ? (p1 + 2) % 3 : (p1 + 1) % 3;
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            if (td_slice(t, i, j) != want) continue;
            const int32_t f = TD(B, i, j);
            int t1, t4, t16, t64, c;
            if (t == 2) {
                const int32_t n1 = TD(B, i - 1, j), n2 = TD(B, i, j + 1), n3 = TD(B, i + 1, j), n4 = TD(B, i, j - 1);
                c = dg(n1, 2) == 1;
                t1 = dg(f, 0) == 1 ? 1 : 3 * (dg(n1, 2) == 3) + 2 * (dg(n1, 1) == 3);
                t4 = (n2 & 256) ? 2 : (dg(f, 1) != 2) * dg(f, 1);
                t16 = (n3 & 256) ? 1 : (dg(f, 2) != 1) * dg(f, 2);
                t64 = dg(f, 3) == 2 ? 2 : (dg(n4, 2) == 3) + 3 * (dg(n4, 1) == 3);
            } else {
                const int32_t n1 = t == 0 ? TD(B, i - 1, j) : TD(B, i - 1, j + 1);
                const int32_t n2 = t == 0 ? TD(B, i - 1, j + 1) : TD(B, i, j + 1);
                const int32_t n3 = t == 0 ? TD(B, i + 1, j) : TD(B, i + 1, j - 1);
                const int32_t n4 = t == 0 ? TD(B, i + 1, j - 1) : TD(B, i, j - 1);
                c = dg(n3, 0) == 2;
                t1 = (n1 & 256) ? 2 : (dg(f, 0) != 2) * dg(f, 0);
                t4 = (n2 & 256) ? 1 : (dg(f, 1) != 1) * dg(f, 1);
                t16 = dg(f, 2) == 2 ? 2 : 3 * (dg(n3, 0) == 3) + (dg(n3, 1) == 3);
                t64 = dg(f, 3) == 1 ? 1 : 2 * (dg(n4, 0) == 3) + 3 * (dg(n4, 1) == 3);
            }
            TD(B, i, j) = bf_pack(t1, t4, t16, t64, c);
        }
}

/* Pass 23: finishes the slice of pass 21. */
static void td_butterfly_pass23(td_state* st, int32_t* B, int t, int p1) {
    const int want = t == 0 ? (p1 + 1) % 3 : (p1 + 2) % 3;
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            if (td_slice(t, i, j) != want) continue;
            const int32_t f = TD(B, i, j);
            const int c = (f >> 8) & 1;
            int t1 = dg(f, 0), t4 = dg(f, 1), t16 = dg(f, 2), t64 = dg(f, 3);
            if (t == 2) {
                const int32_t n1 = TD(B, i - 1, j), n4 = TD(B, i, j - 1);
                t1 = (n1 & 256) ? 1 : (dg(f, 0) != 1) * dg(f, 0);
                t64 = (n4 & 256) ? 2 : (dg(f, 3) != 2) * dg(f, 3);
            } else {
                const int32_t n3 = t == 0 ? TD(B, i + 1, j) : TD(B, i + 1, j - 1);
                const int32_t n4 = t == 0 ? TD(B, i + 1, j - 1) : TD(B, i, j - 1);
                t16 = (n3 & 256) ? 2 : (dg(f, 2) != 2) * dg(f, 2);
                t64 = (n4 & 256) ? 1 : (dg(f, 3) != 1) * dg(f, 3);
            }
            TD(B, i, j) = bf_pack(t1, t4, t16, t64, c);
        }
}

/* UpdateLozengeFromButterflys{H,L,R} (:655-746). */
static void td_lozenges_from_butterfly(td_state* st, int t) {
    for (int i = 1; i <= st->m - 2; ++i)
        for (int j = 1; j <= st->m - 2; ++j) {
            const int32_t b = t == 0 ? TD(st->BH, i, j) : t == 1 ? TD(st->BL, i, j) : TD(st->BR, i, j);
            const int d0 = dg(b, 0), d1 = dg(b, 1), d2 = dg(b, 2), d3 = dg(b, 3), c = (b >> 8) & 1;
            const int32_t own = (d0 == 3) + 2 * (d1 == 3) + 4 * (d2 == 3) + 8 * (d3 == 3);
            if (t == 0) {
                TD(st->H, i, j) = own;
                TD(st->L, i, j) = c + 2 * (d2 == 3) + 4 * (d3 == 1) + 8 * (d3 == 2);
                TD(st->R, i, j) = c + 2 * (d2 == 1) + 4 * (d2 == 2) + 8 * (d3 == 3);
            } else if (t == 1) {
                TD(st->L, i, j) = own;
                TD(st->R, i, j) = (d0 == 3) + 2 * (d1 == 1) + 4 * (d1 == 2) + 8 * c;
                TD(st->H, i, j) = (d0 == 1) + 2 * (d0 == 2) + 4 * (d1 == 3) + 8 * c;
            } else {
                TD(st->R, i, j) = own;
                TD(st->H, i, j) = (d0 == 1) + 2 * (d0 == 2) + 4 * c + 8 * (d3 == 3);
                TD(st->L, i, j) = (d0 == 3) + 2 * c + 4 * (d3 == 1) + 8 * (d3 == 2);
            }
        }
}

/* TilingToTriangleFlips / TilingToButterflyFlips (TriangleDimerTiler.cpp:634-709):
 * the derived arrays the host builds before a walk. */
static void td_derive(const int32_t* t, int n, int32_t* tri, int32_t* bfl) {
#define T(i, j) t[(int64_t)(i) * n + (j)]
    for (int64_t k = 0; k < (int64_t)(n / 2) * n; ++k) tri[k] = 0;
    for (int64_t k = 0; k < (int64_t)n * n; ++k) bfl[k] = 0;
    for (int i = 1; i < n / 2 - 1; ++i)
        for (int j = 1; j < n - 1; ++j) {
            const int32_t a = T(2 * i + 1, j), b = T(2 * i + 1, j + 1);
            int32_t v;
            if (j % 2 == 0) {
                const int32_t c = T(2 * i, j + 1);
                v = (((a >> 2) & 1) + ((a >> 2) & 2) + 3 * ((b >> 3) & 1)) +
                    4 * (((b >> 2) & 1) + (a & 2) + 3 * ((b >> 1) & 1)) +
                    16 * (2 * (c & 1) + (a & 1) + 3 * ((c >> 1) & 1));
            } else {
                const int32_t c = T(2 * i + 2, j);
                v = ((a & 1) + ((a >> 2) & 2) + 3 * ((b >> 3) & 1)) + 4 * ((b & 1) + (a & 2) + 3 * ((b >> 1) & 1)) +
                    16 * (((c >> 2) & 2) + 3 * ((c >> 2) & 1) + ((a >> 2) & 1));
            }
            tri[(int64_t)i * n + j] = v;
        }
    for (int i = 2; i < n - 2; ++i)
        for (int j = 2; j < n - 2; ++j) {
            int f1, f4, f16, f64, c;
            const int32_t x = T(i, j);
            if (i % 2 == 0) {
                if (j % 2 == 0) continue;
                const int32_t u = T(i - 1, j), ue = T(i - 1, j + 1), d = T(i + 1, j), dw = T(i + 1, j - 1);
                f1 = ((u >> 3) & 1) + 2 * (u & 1) + 3 * (x & 1);
                f4 = (ue & 1) + (ue & 2) + 3 * ((x >> 1) & 1);
                f16 = ((d >> 1) & 1) + ((d >> 1) & 2) + 3 * ((x >> 2) & 1);
                f64 = ((dw >> 2) & 1) + ((dw >> 2) & 2) + 3 * ((x >> 3) & 1);
                c = (ue >> 2) & 1;
            } else if (j % 2 == 0) {
                const int32_t ue = T(i - 1, j + 1), e = T(i, j + 1), dw = T(i + 1, j - 1), w = T(i, j - 1);
                f1 = (ue & 1) + (ue & 2) + 3 * (x & 1);
                f4 = ((e >> 1) & 1) + ((e >> 1) & 2) + 3 * ((x >> 1) & 1);
                f16 = ((dw >> 2) & 1) + ((dw >> 2) & 2) + 3 * ((x >> 2) & 1);
                f64 = ((w >> 3) & 1) + 2 * (w & 1) + 3 * ((x >> 3) & 1);
                c = (e >> 3) & 1;
            } else {
                const int32_t u = T(i - 1, j), e = T(i, j + 1), d = T(i + 1, j), w = T(i, j - 1);
                f1 = (u & 1) + (u & 2) + 3 * (x & 1);
                f4 = (e & 1) + (e & 2) + 3 * ((x >> 1) & 1);
                f16 = ((d >> 2) & 1) + ((d >> 2) & 2) + 3 * ((x >> 2) & 1);
                f64 = ((w >> 2) & 1) + ((w >> 2) & 2) + 3 * ((x >> 3) & 1);
                c = (e >> 3) & 1;
            }
            bfl[(int64_t)i * n + j] = f1 + 4 * f4 + 16 * f16 + 64 * f64 + 256 * c;
        }
#undef T
}

static int tridimer_run(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                        int fast, uint32_t chain) {
    if (n < 8 || n % 2) return ORC_EINVAL;
    const int m = n / 2;
    const size_t mm = (size_t)m * m;
    int32_t* buf = (int32_t*)calloc(8 * mm, sizeof(int32_t));
    int32_t* tri = (int32_t*)calloc((size_t)(n / 2) * n, sizeof(int32_t));
    int32_t* bfl = (int32_t*)calloc((size_t)n * n, sizeof(int32_t));
    if (!buf || !tri || !bfl) {
        free(buf);
        free(tri);
        free(bfl);
        return ORC_ENOMEM;
    }
    td_state S = {m, buf, buf + mm, buf + 2 * mm, buf + 3 * mm, buf + 4 * mm, buf + 5 * mm, buf + 6 * mm, buf + 7 * mm};
    td_state* st = &S;
    td_derive(t, n, tri, bfl);
    /* Split (TriangleDimerTiler.cpp:107-133). */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const int64_t at = (int64_t)(i / 2) * m + j / 2;
            if (i % 2 == 0) {
                if (j % 2 == 1) S.H[at] = t[(int64_t)i * n + j], S.BH[at] = bfl[(int64_t)i * n + j];
            } else if (j % 2 == 0) {
                S.L[at] = t[(int64_t)i * n + j], S.BL[at] = bfl[(int64_t)i * n + j];
            } else {
                S.R[at] = t[(int64_t)i * n + j], S.BR[at] = bfl[(int64_t)i * n + j];
            }
        }
    for (int i = 0; i < n / 2; ++i)
        for (int j = 0; j < n; ++j) (j % 2 == 0 ? S.D : S.U)[(int64_t)i * m + j / 2] = tri[(int64_t)i * n + j];
    orc_draws draws, *rng = &draws;
    int err = draws_begin(rng, fast, (int64_t)mm, m, 0, 0, m, fast ? (uint64_t)seed : (uint32_t)(uint64_t)seed, chain,
                          params, nparams);
    if (err == ORC_OK) {
        minstd g;
        minstd_seed(&g, seed);
        int32_t* lz[3] = {S.H, S.L, S.R};
        int32_t* bf[3] = {S.BH, S.BL, S.BR};
        for (int64_t s = 0; s < steps; ++s) {
            /* Fast mode: step s makes move s mod 30 of a fixed sweep over every
             * flip class -- lozenges (orientation r1, class r2), triangles
             * (kind r2, class r1), butterflies (orientation r1, slice p1,
             * parity p2) -- instead of drawing the move. */
            int kind, r1, r2, p1 = 0, p2 = 0;
            if (fast) {
                const int mv = (int)(s % 30);
                if (mv < 6) {
                    kind = 0, r1 = mv / 2, r2 = mv % 2;
                } else if (mv < 12) {
                    kind = 1, r2 = (mv - 6) / 3, r1 = (mv - 6) % 3;
                } else {
                    kind = 2, r1 = (mv - 12) / 6, p1 = ((mv - 12) / 2) % 3, p2 = (mv - 12) % 2;
                }
            } else {
                kind = uniform_int(&g, 2), r1 = uniform_int(&g, 2), r2 = uniform_int(&g, 1);
            }
            if (kind == 0) { /* lozenge flips, TriangleDimerTiler.cpp:243-278 */
                td_rotate_lozenges(st, lz[r1], r1, r2, rng);
                td_lozenges_flipped(st, lz[r1], r1, r2);
                td_lozenges_other(st, r1);
                td_up_from_lozenges(st);
                td_triangles_other(st, S.U, S.D, 0);
                for (int w = 0; w < 3; ++w) td_butterfly_from_lozenges(st, w);
            } else if (kind == 1) { /* triangle flips, :279-305 */
                int32_t* A = r2 == 1 ? S.D : S.U;
                td_rotate_triangles(st, A, r1, rng);
                td_triangles_flipped(st, A, r2 == 0, r1);
                if (r2 == 1)
                    td_triangles_other(st, S.D, S.U, 1);
                else
                    td_triangles_other(st, S.U, S.D, 0);
                td_lozenges_from_triangles(st);
                for (int w = 0; w < 3; ++w) td_butterfly_from_lozenges(st, w);
            } else { /* butterfly flips, :306-347 */
                if (!fast) p1 = uniform_int(&g, 2), p2 = uniform_int(&g, 1);
                td_rotate_butterflies(st, bf[r1], r1, p1, p2, rng);
                td_butterfly_same_slice(st, bf[r1], r1, p1, p2);
                td_butterfly_pass21(st, bf[r1], r1, p1);
                td_butterfly_pass22(st, bf[r1], r1, p1);
                td_butterfly_pass23(st, bf[r1], r1, p1);
                td_lozenges_from_butterfly(st, r1);
                for (int w = 0; w < 3; ++w)
                    if (w != r1) td_butterfly_from_lozenges(st, w);
                td_up_from_lozenges(st);
                td_triangles_other(st, S.U, S.D, 0);
            }
            draws_next(rng);
        }
        draws_end(rng);
        /* Only the lozenge states go back into the tiling (:362-376). */
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const int64_t at = (int64_t)(i / 2) * m + j / 2;
                if (i % 2 == 0) {
                    if (j % 2 == 1) t[(int64_t)i * n + j] = S.H[at];
                } else {
                    t[(int64_t)i * n + j] = j % 2 == 0 ? S.L[at] : S.R[at];
                }
            }
    }
    free(buf);
    free(tri);
    free(bfl);
    return err;
}

/* The eight state arrays of a tiling, m x m each (m = n / 2), in the order
 * H, L, R, U, D, BH, BL, BR: the split of TriangleDimerTiler.cpp:107-133 as
 * tridimer_run performs it. */
int orc_tridimer_arrays(const int32_t* t, int n, int32_t* out8) {
    if (n < 8 || n % 2 || !t || !out8) return ORC_EINVAL;
    const int m = n / 2;
    const size_t mm = (size_t)m * m;
    int32_t* tri = (int32_t*)calloc((size_t)(n / 2) * n, sizeof(int32_t));
    int32_t* bfl = (int32_t*)calloc((size_t)n * n, sizeof(int32_t));
    if (!tri || !bfl) {
        free(tri);
        free(bfl);
        return ORC_ENOMEM;
    }
    td_derive(t, n, tri, bfl);
    int32_t *H = out8, *L = out8 + mm, *R = out8 + 2 * mm, *U = out8 + 3 * mm, *D = out8 + 4 * mm;
    int32_t *BH = out8 + 5 * mm, *BL = out8 + 6 * mm, *BR = out8 + 7 * mm;
    for (size_t e = 0; e < 8 * mm; ++e) out8[e] = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const int64_t at = (int64_t)(i / 2) * m + j / 2;
            if (i % 2 == 0) {
                if (j % 2 == 1) H[at] = t[(int64_t)i * n + j], BH[at] = bfl[(int64_t)i * n + j];
            } else if (j % 2 == 0) {
                L[at] = t[(int64_t)i * n + j], BL[at] = bfl[(int64_t)i * n + j];
            } else {
                R[at] = t[(int64_t)i * n + j], BR[at] = bfl[(int64_t)i * n + j];
            }
        }
    for (int i = 0; i < n / 2; ++i)
        for (int j = 0; j < n; ++j) (j % 2 == 0 ? D : U)[(int64_t)i * m + j / 2] = tri[(int64_t)i * n + j];
    free(tri);
    free(bfl);
    return ORC_OK;
}

int orc_tridimer_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams) {
    return tridimer_run(t, n, steps, seed, params, nparams, 0, 0);
}

int orc_tridimer_walk_fast(int32_t* t, int n, int64_t steps, int64_t key, uint32_t chain) {
    return tridimer_run(t, n, steps, key, NULL, 0, 1, chain);
}

/* ------------------------------------------------------------------------ */
/* Height-function projection (no reference counterpart; the checker of    */
/* rt_project_heights).  Graph: DominoTiler::DomainToVertices               */
/* (DominoTiler.cpp:479-500) / LozengeTiler::DomainToVertices               */
/* (LozengeTiler.cpp:405-434) for the vertex kinds, and the edges           */
/* TilingToHeightfunc walks (DominoTiler.cpp:204-206,423-458;               */
/* LozengeTiler.cpp:12-16,95-138): neighbour inside and one of the two      */
/* faces beside the edge in the domain.  Edge step s: dominoes              */
/* (nb > 1 ? 1 : -1) * ((i+j) even ? 1 : -1), lozenges dh[nb].              */
/* ------------------------------------------------------------------------ */
static const int kPDomN[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
static const int kPDomF[4][2][2] = {{{0, -1}, {0, 0}}, {{-1, -1}, {-1, 0}}, {{-1, 0}, {0, 0}}, {{-1, -1}, {0, -1}}};
static const int kPLozN[6][2] = {{0, 1}, {-1, 1}, {-1, 0}, {0, -1}, {1, -1}, {1, 0}};
static const int kPLozS[6] = {-1, 1, -1, 1, -1, 1};
static const int kPLozF[6][2][2] = {{{0, 0}, {-1, 1}}, {{-1, 1}, {-1, 0}}, {{-1, 0}, {-1, -1}},
                                    {{-1, -1}, {0, -2}}, {{0, -2}, {0, -1}}, {{0, -1}, {0, 0}}};

static int p_dface(const int32_t* d, int m, int i, int j) { return i >= 0 && j >= 0 && i < m && j < m ? d[i * m + j] != 0 : 0; }
static int p_lface(const int32_t* d, int m, int r, int c) {
    return r >= 0 && c >= 0 && r < m && c < 2 * m ? d[r * 2 * m + c] != 0 : 0;
}

int orc_project_heights(int model, const int32_t* d, int64_t dlen, const int32_t* hmin, const int32_t* hmax,
                        const float* target, int32_t* out, int n, int64_t* passes_out) {
    const int dom = model == 0;
    const int m = n - 1;
    if ((dom && (int64_t)m * m != dlen) || (!dom && (int64_t)2 * m * m != dlen) || m < 2) return ORC_EINVAL;
    const int nb_count = dom ? 4 : 6, M = dom ? 4 : 3;
    uint8_t* kind = (uint8_t*)calloc((size_t)n * n, 1);
    uint8_t* edges = (uint8_t*)calloc((size_t)n * n, 1);
    if (!kind || !edges) {
        free(kind);
        free(edges);
        return ORC_ENOMEM;
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            int k = 0;
            if (dom) {
                if (i == 0 || j == 0 || i == m || j == m) {
                    const int i0 = i - (i == m), i1 = i - 1 + (i == 0), j0 = j - (j == m), j1 = j - 1 + (j == 0);
                    if (p_dface(d, m, i0, j0) || p_dface(d, m, i1, j0) || p_dface(d, m, i0, j1) || p_dface(d, m, i1, j1))
                        k = 2;
                } else {
                    const int c = p_dface(d, m, i - 1, j - 1) + p_dface(d, m, i - 1, j) + p_dface(d, m, i, j - 1) +
                                  p_dface(d, m, i, j);
                    k = c == 4 ? 1 : c > 0 ? 2 : 0;
                }
            } else if (!(i == 0 || j == 0 || i == m || j == m)) {
                const int c = p_lface(d, m, i, 2 * j) + p_lface(d, m, i, 2 * j - 1) + p_lface(d, m, i, 2 * j - 2) +
                              p_lface(d, m, i - 1, 2 * j) + p_lface(d, m, i - 1, 2 * j + 1) + p_lface(d, m, i - 1, 2 * j - 1);
                k = c == 6 ? 1 : c > 0 ? 2 : 0;
            }
            kind[i * n + j] = (uint8_t)k;
        }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            if (!kind[i * n + j]) continue;
            for (int nb = 0; nb < nb_count; ++nb) {
                const int i2 = i + (dom ? kPDomN[nb][0] : kPLozN[nb][0]), j2 = j + (dom ? kPDomN[nb][1] : kPLozN[nb][1]);
                if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n || !kind[i2 * n + j2]) continue;
                int in;
                if (dom)
                    in = p_dface(d, m, i + kPDomF[nb][0][0], j + kPDomF[nb][0][1]) ||
                         p_dface(d, m, i + kPDomF[nb][1][0], j + kPDomF[nb][1][1]);
                else
                    in = p_lface(d, m, i + kPLozF[nb][0][0], 2 * j + kPLozF[nb][0][1]) ||
                         p_lface(d, m, i + kPLozF[nb][1][0], 2 * j + kPLozF[nb][1][1]);
                if (in) edges[i * n + j] |= (uint8_t)(1u << nb);
            }
        }
    /* 1. residue rounding, clamped; boundary vertices fixed at h_min */
    for (int64_t v = 0; v < (int64_t)n * n; ++v) {
        if (!kind[v]) {
            out[v] = INT32_MAX;
        } else if (kind[v] == 2) {
            out[v] = hmin[v];
        } else {
            const double q = floor(((double)target[v] - (double)hmin[v]) / (double)M + 0.5);
            double g = (double)hmin[v] + (double)M * q;
            if (g < (double)hmin[v]) g = (double)hmin[v];
            if (g > (double)hmax[v]) g = (double)hmax[v];
            out[v] = (int32_t)g;
        }
    }
    /* 2. min-plus relaxation of the interior vertices, in place, until a pass changes nothing */
    int64_t passes = 0;
    int changed = 1;
    while (changed) {
        changed = 0;
        ++passes;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const int64_t v = (int64_t)i * n + j;
                if (kind[v] != 1) continue;
                int32_t best = out[v];
                for (int nb = 0; nb < nb_count; ++nb) {
                    if (!(edges[v] & (1u << nb))) continue;
                    const int i2 = i + (dom ? kPDomN[nb][0] : kPLozN[nb][0]), j2 = j + (dom ? kPDomN[nb][1] : kPLozN[nb][1]);
                    const int s = dom ? (nb > 1 ? 1 : -1) * (((i + j) % 2 == 0) ? 1 : -1) : kPLozS[nb];
                    const int32_t cand = out[(int64_t)i2 * n + j2] + (s == -1 ? 1 : M - 1);
                    if (cand < best) best = cand;
                }
                if (best < out[v]) {
                    out[v] = best;
                    changed = 1;
                }
            }
    }
    /* 3. back up to h_min */
    for (int64_t v = 0; v < (int64_t)n * n; ++v)
        if (kind[v] && out[v] < hmin[v]) out[v] = hmin[v];
    if (passes_out) *passes_out = passes;
    free(kind);
    free(edges);
    return ORC_OK;
}
