/* rt_b200.h -- C ABI of the B200 flip-dynamics engine (librt_b200.so).
 *
 * This is the drop-in boundary for RandomTilings' per-model Tiler classes.
 * Each entry point names the reference interface it replaces (paths are
 * relative to the GPUTilings/RandomTilings source tree).  Plain pointers and
 * sizes only; every function returns an rt_status (0 = success) and never
 * throws or exits.  Tilings are host int32 arrays of N x N, row-major, in the
 * reference's encodings:
 *   domino        src/Domino/DominoTiler.h:17-37       (vertex edge bits)
 *   lozenge       src/Lozenge/LozengeTiler.h:8-28       (vertex edge bits)
 *   rect-triangle src/RectTriangle/RectTriangleTiler.h:16-27 (hex face digits)
 *   tri-dimer     src/TriangleDimer/TriangleDimerTiler.h:13-67 (lozenge states)
 * A handle (rt_tiler) is not thread-safe, like the reference classes, which
 * own one command queue and one RNG buffer each.
 */
#ifndef RT_B200_H
#define RT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    RT_OK = 0,
    RT_E_INVAL = -1,     /* bad argument or tiling size */
    RT_E_PARAMS = -2,    /* TinyMT parameter table missing, short or malformed */
    RT_E_NOMEM = -3,     /* device or host allocation failed */
    RT_E_CUDA = -4,      /* a CUDA call failed (rt_last_error has the text) */
    RT_E_TIMEOUT = -5,   /* a bounded device wait gave up (kernel returned early) */
    RT_E_NODEVICE = -6,  /* no usable sm_100 device */
    RT_E_STATE = -7      /* call out of order (e.g. run before upload) */
} rt_status;

typedef enum { RT_DOMINO = 0, RT_LOZENGE = 1, RT_RECTTRI = 2, RT_TRIDIMER = 3 } rt_model;

/* Which reference kernel file the flip follows. */
typedef enum {
    RT_KERNEL_DEFAULT = 0, /* dominokernel.cl / lozengekernel.cl / recttrianglekernel.cl / triangledimerkernel.cl */
    RT_KERNEL_CFTP = 1,    /* domino only: dominokernelCFTP.cl (monotone heat bath) */
    RT_KERNEL_QWEIGHT = 2  /* lozenge only: qlozengekernel.cl (volume weight q, int32 storage) */
} rt_kernel;

typedef enum {
    RT_RNG_TINYMT = 0, /* bit-exact: per-work-item TinyMT streams + the reference's host colour order */
    RT_RNG_PHILOX = 1, /* fast mode: Philox4x32-10 keyed by (chain, site, sweep, colour), cyclic colour sweeps */
    RT_RNG_PLANES = 2  /* bit-plane mode (dominoes; uniform lozenges): the lattice as bit planes, 32 sites per
                          word, one Philox4x32-10 bit per site and colour step, cyclic colour sweeps.  Rules:
                          domino heat bath (RT_KERNEL_CFTP): a rotatable site becomes 12 where its bit is 1,
                          else 3; domino toggle (RT_KERNEL_DEFAULT): 3 <-> 12 where either of two bits is 1
                          (probability 3/4 instead of dominokernel.cl's 0.8); lozenges: heat bath, 25 -> 38
                          where the bit is 1, 38 -> 25 where it is 0.  Same equilibrium (uniform); the heat
                          baths are monotone, so rt_cftp accepts them. */
} rt_rng;

typedef enum {
    RT_QCMP_FLOAT32 = 0, /* q rounded to float before the compare (an fp32-only OpenCL device) */
    RT_QCMP_DOUBLE = 1   /* q compared as the double literal of qlozengekernel.cl:3 */
} rt_qcmp;

typedef struct {
    int32_t model;       /* rt_model */
    int32_t kernel;      /* rt_kernel */
    int32_t rng;         /* rt_rng */
    int32_t qcmp;        /* rt_qcmp, q-weighted lozenge only */
    double q;            /* volume weight, qlozengekernel.cl:3 (0.99) */
    float weights[16];   /* rect-triangle face weights by digit, recttrianglekernel.cl:3-13 */
    int32_t device;      /* CUDA device ordinal */
    uint32_t chain;      /* fast mode: Philox counter word 3 (a chain's index in a batch); 0 otherwise */
    void* stream;        /* cudaStream_t to run on; NULL = the handle creates its own */
} rt_config;

typedef struct rt_tiler rt_tiler;

/* Fills *cfg with the reference defaults (q = 0.99, unit weights, TinyMT). */
void rt_config_default(rt_config* cfg, int32_t model);

/* Replaces the constructors DominoTiler(context, queue, devices, source, err)
 * src/Domino/DominoTiler.h:61-67, LozengeTiler src/Lozenge/LozengeTiler.h:47-53,
 * RectTriangleTiler src/RectTriangle/RectTriangleTiler.h:45-52 and
 * TriangleDimerTiler src/TriangleDimer/TriangleDimerTiler.h:116-174.  The
 * OpenCL objects become a device ordinal (+ optional stream) in *cfg. */
rt_status rt_create(const rt_config* cfg, rt_tiler** out);
rt_status rt_destroy(rt_tiler* h);

/* Replaces LoadTinyMT(std::string params, int size), e.g.
 * src/Domino/DominoTiler.cpp:109-111 -> src/TinyMT/file_reader.cpp:22-38.
 * Reads `n` (mat1, mat2, tmat) triples from a tinymt32dc text table.  With no
 * table loaded, every work item uses the TinyMT32J constants
 * (src/TinyMT/tinymt32def.h:47-49). */
rt_status rt_load_rng_params(rt_tiler* h, const char* path, int64_t n);
/* Same, from memory: 3*n uint32 (mat1, mat2, tmat per id). */
rt_status rt_set_rng_params(rt_tiler* h, const uint32_t* table, int64_t n);

/* Weighted dominoes (no reference counterpart; the reference's heat-bath
 * kernel dominokernelCFTP.cl:19-28 is the uniform case): the heat-bath
 * kernel (RT_KERNEL_CFTP) with periodic domino weights.  A domino covering
 * squares (r, c) and (r, c+1) weighs wh[(r mod P) P + (c mod P)], one
 * covering (r, c) and (r+1, c) wv[(r mod P) P + (c mod P)] (square (r, c)
 * spans vertices (r..r+1, c..c+1)); period P is 1, 2 or 4, weights finite
 * and > 0.  At a rotatable vertex (i, j) the two horizontal dominoes (state
 * 3) weigh w3 = wh(i-1, j-1) wh(i, j-1) and the two vertical ones (state 12)
 * w12 = wv(i-1, j-1) wv(i-1, j); the site becomes 12 when the draw is below
 * w12 / (w3 + w12), else 3 -- for equal weights exactly the reference's
 * 0.5.  The walk, epoch walk and CFTP of the handle use them in the TinyMT
 * and Philox modes; RT_RNG_PLANES (one random bit per site) rejects them.
 * period = 0 returns to uniform weights. */
rt_status rt_set_domino_weights(rt_tiler* h, int32_t period, const double* wh, const double* wv);

/* Weighted lozenges (no reference counterpart; lozengekernel.cl:19-31 is
 * the uniform case): the uniform-lozenge kernel (char storage) with
 * periodic lozenge weights.  A lozenge is weighed by the lattice edge it
 * covers, named by its lower end (i, j): w0 for the edge to (i, j+1) (bit
 * 8), w1 for (i-1, j+1) (bit 2), w2 for (i-1, j) (bit 1), each table
 * indexed [(i mod P) P + (j mod P)], P = 1, 2 or 4, weights finite and
 * > 0.  At a flippable vertex (i, j), state 25 weighs
 * W25 = w2(i, j) w0(i, j) w1(i+1, j-1) and state 38
 * W38 = w1(i, j) w0(i, j-1) w2(i+1, j); with p = W38 / (W25 + W38) a draw
 * below 0.8 p turns 25 into 38 and one in [0.8 p, 0.8) turns 38 into 25 --
 * for equal weights exactly the reference's 0.4 / 0.8.  Walks, epoch walks
 * and CFTP of the handle use them in the TinyMT and Philox modes;
 * RT_RNG_PLANES rejects them.  period = 0 returns to uniform weights. */
rt_status rt_set_lozenge_weights(rt_tiler* h, int32_t period, const double* w0, const double* w1, const double* w2);

/* Replaces Walk(tiling&, long steps, long seed) src/Domino/DominoTiler.cpp:9-55,
 * Walk(tiling&, int, long) src/Lozenge/LozengeTiler.cpp:18-88,
 * src/RectTriangle/RectTriangleTiler.cpp:17-92,
 * src/TriangleDimer/TriangleDimerTiler.cpp:86-483.  `tiling` (N*N int32,
 * host) is updated in place; synchronous, like the reference.  A call (and
 * each rt_walk_epochs / rt_run / CFTP trial, all epochs together) takes at
 * most 2^40 steps; more is RT_E_INVAL, with the tiling left as it was.
 * Tiling sides above 32767 are RT_E_INVAL (the kernels' indices are 32-bit). */
rt_status rt_walk(rt_tiler* h, int32_t* tiling, int32_t n, int64_t steps, int64_t seed);

/* Replaces DominoTiler::Walk(tiling&, vector<long> steps, vector<long> seeds)
 * src/Domino/DominoTiler.cpp:58-107 (k epochs, TinyMT re-seeded each epoch). */
rt_status rt_walk_epochs(rt_tiler* h, int32_t* tiling, int32_t n, const int64_t* steps, const int64_t* seeds,
                         int32_t k);

/* Coupling from the past on a monotone chain: the domino heat bath (handle
 * created with RT_KERNEL_CFTP) or either lozenge kernel (epochs restart the
 * colour engine and the draws from the epoch seed, as the domino epoch Walk
 * does); in fast mode (RT_RNG_PHILOX) each epoch seed is that epoch's Philox
 * key.  Replaces the driver of Examples/AztecDiamondCftpEx.cpp:42-68
 * over DominoTiler::Walk(tiling&, vector<long>, vector<long>)
 * (src/Domino/DominoTiler.cpp:58-107): both chains (from tmax and tmin) run
 * through the same epochs as two coupled lattices of one launch and are
 * compared on the device.  Epoch seeds are successive std::mt19937(master_seed)
 * outputs, newest epoch first.  schedule = RT_CFTP_REFERENCE prepends
 * 2 * first_steps each trial (the example's +256 with first_steps = 128);
 * RT_CFTP_DOUBLING doubles the total.  out_tiling (optional) receives the
 * coalesced tiling. */
typedef enum { RT_CFTP_DOUBLING = 0, RT_CFTP_REFERENCE = 1 } rt_cftp_schedule;
typedef struct {
    int64_t total_steps; /* colour steps from the past of the last trial */
    int32_t trials;      /* trials run */
    int32_t coalesced;   /* 1 if the chains met within max_trials */
    double device_ms;    /* device time of the walks of all trials */
} rt_cftp_stats;
rt_status rt_cftp(rt_tiler* h, const int32_t* tmax, const int32_t* tmin, int32_t n, int64_t first_steps,
                  int32_t schedule, int64_t master_seed, int32_t max_trials, int32_t* out_tiling,
                  rt_cftp_stats* stats);

/* Split form of rt_walk, for callers that keep the lattice on the device
 * (the reference re-uploads per Walk, DominoTiler.cpp:26-27,46-47):
 * upload + split into colour arrays, run steps (asynchronous on the handle's
 * stream), merge + download.  rt_walk == upload; run; download. */
rt_status rt_upload(rt_tiler* h, const int32_t* tiling, int32_t n);
rt_status rt_run(rt_tiler* h, int64_t steps, int64_t seed);
rt_status rt_download(rt_tiler* h, int32_t* tiling);
rt_status rt_synchronize(rt_tiler* h);
/* The handle's cudaStream_t (as void*), for callers that time with events. */
void* rt_stream(rt_tiler* h);
/* Device form of rt_download, for statistics computed on the device (no
 * reference counterpart): merges the colour arrays into the handle's own
 * N x N int32 device tiling (asynchronous on rt_stream(h)) and returns its
 * address in *d_tiling; it stays valid until the next rt_upload / rt_walk
 * or rt_destroy, and is overwritten by the next rt_download / rt_device_tiling. */
rt_status rt_device_tiling(rt_tiler* h, int32_t** d_tiling);
/* Counters of the last run: phases executed and kernel launches issued. */
rt_status rt_last_run_info(rt_tiler* h, int64_t* phases, int64_t* launches);

/* No counterpart in the reference.  For callers that may not allocate GPU
 * memory through the library -- programs that hand out all device memory
 * from their own fixed pool, where a cudaMalloc/cudaFree inside a library
 * would break their accounting and synchronise the device.  Same walk as
 * rt_walk (TinyMT32J parameters, reference colour order), but `d_tiling` is
 * the caller's DEVICE buffer (N*N int32, in and out) and no handle exists:
 * every other byte the walk needs sits in one built-in device array of
 * 16 MiB per GPU, kept until the process exits.  Walks that need more
 * (tiling side x steps) are rejected with RT_E_INVAL.  Calls share the
 * array: calls that overlap on one GPU race.  Runs on cfg->stream (NULL =
 * the default stream) and returns after the walk has finished there: the
 * call is synchronous and must not be made while that stream is being
 * captured into a graph.  The tiling is written back only after a walk that
 * finished: after RT_E_INVAL or RT_E_TIMEOUT it holds its input unchanged.
 * A failure message goes to errbuf (errcap bytes) when errbuf is not NULL. */
rt_status rt_walk_device_noalloc(const rt_config* cfg, int32_t* d_tiling, int32_t n, int64_t steps, int64_t seed,
                                 char* errbuf, size_t errcap);

/* Text of the last failure on this handle (or of the last rt_create). */
const char* rt_last_error(rt_tiler* h);
const char* rt_version(void);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_H */
