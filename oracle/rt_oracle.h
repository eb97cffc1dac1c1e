/* rt_oracle.h -- CPU restatement of RandomTilings' flip dynamics.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA product is compared
 * against: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it.  The product library never links it.
 *
 * Parity of this restatement is pinned against the reference's own code
 * (oracle/_ref/libref.so: the reference kernels and Tiler classes compiled unmodified
 * through oracle/shim) by tests/test_oracle_pins.py and the golden fixtures in
 * tests/golden/.
 *
 * Conventions shared by every walk:
 *   - tilings are int32 N x N, row-major, exactly the reference's `tiling`;
 *   - `params` is the TinyMT parameter table, 3 uint32 per work-item id
 *     (mat1, mat2, tmat); NULL means the TinyMT32J constants for every id
 *     (src/TinyMT/tinymt32def.h:47-49);
 *   - return 0 on success, a negative ORC_E* code otherwise.
 */
#ifndef RT_ORACLE_H
#define RT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_OK = 0,
    ORC_EINVAL = -1,   /* bad size / argument */
    ORC_EPARAMS = -2,  /* parameter table too short */
    ORC_ENOMEM = -3
};

/* q-lozenge acceptance arithmetic: qlozengekernel.cl:25 compares the double
 * literal q against a float; an fp32-only device rounds q to float first. */
enum { ORC_QCMP_FLOAT32 = 0, ORC_QCMP_DOUBLE = 1 };

/* ---- generators (exposed for unit tests) ---- */
typedef struct {
    uint32_t s0, s1, s2, s3, mat1, mat2, tmat;
} orc_tinymt;
void orc_tinymt_init(orc_tinymt* st, uint32_t seed);
uint32_t orc_tinymt_bits12(orc_tinymt* st);  /* raw float bits in [1,2) */
float orc_tinymt_single01(orc_tinymt* st);

/* std::mt19937 outputs; std::default_random_engine (minstd_rand0) with
 * std::uniform_int_distribution<int>(0, hi) as libstdc++ implements it. */
void orc_mt19937_stream(int64_t seed, int64_t n, uint32_t* out);
void orc_minstd_raw_stream(int64_t seed, int64_t n, uint32_t* out);
void orc_minstd_uniform_stream(int64_t seed, int64_t n, const int* his, int nhis, int* out);

/* ---- walks ---- */
int orc_domino_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                    int cftp_kernel);
int orc_domino_walk_epochs(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k,
                           const uint32_t* params, int64_t nparams, int cftp_kernel);
/* qmode: 0 = uniform (lozengekernel.cl, char storage); 1 = q-weighted
 * (qlozengekernel.cl, int storage) with comparison `qcmp`; 2 = the batched
 * chains' volume weight on char storage (no reference counterpart): add a
 * cube when rd < 0.4 q, remove one when 0.4 <= rd < 0.8 (double compare). */
int orc_lozenge_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                     int qmode, double q, int qcmp);
/* weights: 16 floats indexed by face digit (recttrianglekernel.cl:3-13);
 * NULL = the reference's all-ones table. */
int orc_recttri_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams,
                     const float* weights);
int orc_tridimer_walk(int32_t* t, int n, int64_t steps, int64_t seed, const uint32_t* params, int64_t nparams);
/* The eight triangle-dimer state arrays (H, L, R, U, D, BH, BL, BR; m x m
 * each, m = n / 2) of a tiling, as the walks split it. */
int orc_tridimer_arrays(const int32_t* t, int n, int32_t* out8);

/* Epoch walks of the lozenge models (each epoch restarts the colour engine
 * and the TinyMT streams from seeds[e], as the domino epoch Walk does). */
int orc_lozenge_walk_epochs(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k,
                            const uint32_t* params, int64_t nparams, int qmode, double q, int qcmp);
/* Weighted lozenges (no reference counterpart; rt_set_lozenge_weights): the
 * uniform rule with the add threshold 0.4 replaced at vertex (i, j) by
 * 0.8 W38 / (W25 + W38) from period x period tables w0, w1, w2 of the
 * lozenges covering the edge from (i, j) to (i, j+1), (i-1, j+1), (i-1, j);
 * fast = 0 TinyMT (epochs as orc_lozenge_walk_epochs), 1 Philox. */
int orc_lozenge_walk_weighted(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k, int fast,
                              uint32_t chain, const uint32_t* params, int64_t nparams, int period, const double* w0,
                              const double* w1, const double* w2);

/* ---- fast mode (no reference counterpart) ----
 * Counter-based draws: Philox4x32-10 keyed by the epoch key, counter =
 * (site word, step within the epoch, chain) -- the site word being the
 * 32-bit word of four consecutive int8 sites of a colour-array row, index
 * i * ceil(width / 4) + j / 4, lane j mod 4; colours in a fixed
 * cycle (dominoes: black, white; three-colour models: 0, 1, 2; triangle
 * dimers: a 30-move sweep over every flip class). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
int orc_domino_walk_fast(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain,
                         int cftp_kernel);
/* Weighted heat bath (no reference counterpart; rt_set_domino_weights):
 * dominokernelCFTP.cl's rule with the threshold 0.5 replaced at vertex (i, j)
 * by w12 / (w3 + w12) from period x period tables of horizontal (wh) and
 * vertical (wv) domino weights indexed by the domino's top-left square.
 * fast = 0: TinyMT draws and the reference's colour order (single_walk as
 * orc_domino_walk, else as orc_domino_walk_epochs); fast = 1: Philox. */
int orc_domino_walk_weighted(int32_t* t, int n, const int64_t* steps, const int64_t* seeds, int k, int single_walk,
                             int fast, uint32_t chain, const uint32_t* params, int64_t nparams, int period,
                             const double* wh, const double* wv);
int orc_lozenge_walk_fast(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain,
                          int qmode, double q, int qcmp);
/* Bit-plane mode (RT_RNG_PLANES): the same colour cycle as fast mode, one
 * Philox bit per site and step (plane_bit in rt_oracle.c), heat-bath rules
 * (dominoes: heat_bath = 1; heat_bath = 0 is the two-bit toggle). */
int orc_domino_walk_planes(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain,
                           int heat_bath);
int orc_lozenge_walk_planes(int32_t* t, int n, const int64_t* steps, const int64_t* keys, int k, uint32_t chain);
int orc_recttri_walk_fast(int32_t* t, int n, int64_t steps, int64_t key, uint32_t chain, const float* weights);
int orc_tridimer_walk_fast(int32_t* t, int n, int64_t steps, int64_t key, uint32_t chain);

/* Exact projection of a real height surface onto a valid height function
 * (the checker of rt_project_heights): model 0 dominoes, 1 lozenges; n the
 * vertex side; hmin / hmax the extremal height functions. */
int orc_project_heights(int model, const int32_t* d, int64_t dlen, const int32_t* hmin, const int32_t* hmax,
                        const float* target, int32_t* out, int n, int64_t* passes);

/* Colour schedules the host loops draw (one entry per step). */
int orc_domino_colours(int64_t seed, int64_t steps, int single_walk, uint8_t* out);
int orc_lozenge_colours(int64_t seed, int64_t steps, uint8_t* out);

/* First step count after which the q-weighted walk differs between the
 * float32 and the double comparison (0: not within max_steps). */
int64_t orc_lozenge_q_divergence(const int32_t* t, int n, int64_t seed, int64_t max_steps, double q);

/* ---- six-vertex model (sixv_oracle.c; no reference code: README.md:3 names
 * the model only).  Heights on the (n+1) x (n+1) faces of an n x n grid with
 * domain-wall boundary conditions; weights w[6] of the vertex types
 * a1, a2, b1, b2, c1, c2; Philox draws as the CUDA walk takes them. ---- */
void orc_sixv_dwbc(int n, int32_t* hmin, int32_t* hmax);
int orc_sixv_vertex_type(int a, int b, int c, int d);
void orc_sixv_thresholds(const double w[6], uint32_t thr[16]);
int orc_sixv_walk(int32_t* h, int n, const int64_t* sweeps, const int64_t* keys, int k, uint32_t chain,
                  const double w[6]);
/* Colour step s of an epoch keyed by `key`, on the face rows [lo, hi) only:
 * what one band of the CUDA band kernel computes (the tests rebuild its
 * halo exchange from it). */
int orc_sixv_step_rows(int32_t* h, int n, int64_t s, uint64_t key, uint32_t chain, const double w[6], int lo,
                       int hi);

#ifdef __cplusplus
}
#endif
#endif /* RT_ORACLE_H */
