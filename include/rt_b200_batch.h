/* rt_b200_batch.h -- many independent chains per launch (fast mode).
 *
 * No reference counterpart: the reference runs one Tiler per lattice and one
 * kernel launch per colour step.  Here any number of chains of any of the
 * four models and of uneven sizes run as ONE CUDA graph holding one
 * persistent launch per kernel family; each launch is a grid of thread-block
 * clusters, a cluster walks whole chains (its CTAs split a chain's rows and
 * exchange halo rows through distributed shared memory), and the chains'
 * lattices stay in shared memory for the whole run.  Draws are the fast mode's
 * (Philox4x32-10, cyclic colours; see rt_b200.h), so chain c with key k gives
 * the tiling that rt_walk gives for a handle created with rng = RT_RNG_PHILOX
 * and chain = c, run with seed k for the same number of colour steps.
 * Cluster size and CTA size per family, and then the number of sweeps one
 * launch runs, are picked by an autotuner that times candidate plans on a
 * scratch copy of the chains (the chains themselves are not advanced).
 */
#ifndef RT_B200_BATCH_H
#define RT_B200_BATCH_H

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rt_batch rt_batch;

typedef struct {
    int32_t model;    /* rt_model */
    int32_t kernel;   /* RT_KERNEL_DEFAULT; dominoes may use RT_KERNEL_CFTP (heat bath) */
    uint32_t chain;   /* Philox counter word 3 */
    float q;          /* lozenges: volume weight q in (0, 1]; 0 = uniform (q = 1).  A site adds a
                         cube when its draw is below 0.4 q and removes one when its draw lies in
                         [0.4, 0.8), so the chain's equilibrium weighs a tiling by q^volume and
                         q = 1 is the uniform rule of lozengekernel.cl:19-21.  Other models: 0. */
    int64_t key;      /* Philox key (the chain's seed) */
} rt_chain;

typedef struct {
    int32_t chains;           /* chains in the batch */
    int32_t cluster[6];       /* per kernel family (domino, domino heat bath, lozenge, -, rect-triangle,
                                 triangle dimer): CTAs per cluster, 0 if the family is absent */
    int32_t block[6];         /* threads per CTA */
    int32_t clusters[6];      /* clusters launched */
    double tune_ms;           /* wall time the autotuner spent */
    double run_ms;            /* device time of the last rt_batch_run (graph launch to end) */
    int64_t attempts;         /* flip attempts in the last rt_batch_run (all chains) */
    int64_t algorithmic_bytes;/* lattice bytes read + written per colour step, summed over the last run */
    int64_t sweeps_per_launch[6]; /* per family: a run of S sweeps is S / this launches (+ one for the rest);
                                     0 = one launch per run */
} rt_batch_info;

rt_status rt_batch_create(int32_t device, rt_batch** out);
rt_status rt_batch_destroy(rt_batch* b);
/* Copies an N x N host tiling into the batch; *index (optional) receives the
 * chain's index.  Chains are added before the first rt_batch_run
 * (RT_E_STATE after it); adding one invalidates the plan.  N above 32767 is
 * RT_E_INVAL. */
rt_status rt_batch_add(rt_batch* b, const rt_chain* c, const int32_t* tiling, int32_t n, int64_t* index);
/* autotune = 1 (default): time the candidate plans at the first run;
 * autotune = 0: use `cluster` CTAs per cluster and `block` threads per CTA
 * for every family (0 = the planner's default); a family whose kernel is
 * built for fewer threads (the triangle dimers': 512) runs with its maximum,
 * which rt_batch_get_info reports. */
rt_status rt_batch_set_tuning(rt_batch* b, int32_t autotune, int32_t cluster, int32_t block);
/* Advances every chain by `sweeps` sweeps: a sweep is every colour (flip
 * class) once -- 2 colour steps for dominoes, 3 for lozenges and
 * rectangle-triangles, 30 for triangle dimers.  Synchronous.  The Philox step
 * counter continues across runs (a run of s1 sweeps then one of s2 equals a
 * run of s1 + s2).  At most 2^35 sweeps per run (and per launch); more is
 * RT_E_INVAL. */
/* Sweeps one launch of a family runs (a run of S sweeps becomes S / sweeps
 * launches plus one for the rest, each continuing the chains' draws), for
 * every family: > 0 fixes it, 0 asks for one launch per run, -1 (the
 * default) lets the autotuner choose. */
rt_status rt_batch_set_sweeps_per_launch(rt_batch* b, int64_t sweeps);
rt_status rt_batch_run(rt_batch* b, int64_t sweeps);
rt_status rt_batch_download(rt_batch* b, int64_t index, int32_t* tiling);
/* Device form of rt_batch_download: chain `index`'s N x N tiling into the
 * caller's device buffer d_tiling (N*N int32), asynchronous on `stream`
 * (cudaStream_t, NULL = the legacy default stream); allocates nothing. */
rt_status rt_batch_device_tiling(rt_batch* b, int64_t index, int32_t* d_tiling, void* stream);
rt_status rt_batch_get_info(rt_batch* b, rt_batch_info* info);
const char* rt_batch_last_error(rt_batch* b);

/* The mixed-domain workload of the batched benchmark, chain `seed` (0, 1,
 * ...): type = seed mod 4 picks the model, sizes come from
 * std::mt19937(seed) through std::uniform_int_distribution<int>:
 *   0: domino, Aztec diamond of order n in [16, 256]           p = {n}
 *   1: lozenge, hexagon with sides a, b, c each in [8, 128]       p = {a, b, c}
 *   2: triangle dimer, bibone hexagon of side 64 with its
 *      canonical start (rt_tridimer_hexagon)                      p = {64}
 *   3: rectangle-triangle, minimal tiling of the side-64 hexagon p = {64}
 * Writes the model to *model and its size parameters to p[0..2]. */
rt_status rt_mixed_chain_spec(int64_t seed, int32_t* model, int32_t* p);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_BATCH_H */
