/* rt_b200_sixv.h -- the six-vertex model (square ice) on the GPU.
 *
 * The reference names the six-vertex model beside its tilings (README.md:3)
 * but ships no code for it; there is no reference interface to replace, so
 * this API follows the reference's Tiler pattern (extremal states, Walk,
 * coupling from the past) on the height-function machinery of the dominoes.
 *
 * State.  An n x n grid of vertices with domain-wall boundary conditions is
 * an integer height function h on the (n+1) x (n+1) faces, row-major int32:
 * h(0,j) = j, h(i,0) = i, h(n,j) = n-j, h(i,n) = n-i, and faces sharing an
 * edge differ by 1.  (h is the corner-sum matrix of an alternating-sign
 * matrix: h = i + j - 2 sum_{k<=i, l<=j} A_kl.)  Vertex (i,j), 1 <= i,j <= n,
 * lies between the faces NW (i-1,j-1), NE (i-1,j), SW (i,j-1), SE (i,j) of
 * heights a, b, c, d; its type is
 *   0 a1: b = a+1, c = a-1, d = a      1 a2: b = a-1, c = a+1, d = a
 *   2 b1: b = c = a+1, d = a+2         3 b2: b = c = a-1, d = a-2
 *   4 c1: b = c = a+1, d = a (A = 1)   5 c2: b = c = a-1, d = a (A = -1)
 * and a configuration weighs the product of its vertices' type weights.
 *
 * Dynamics.  Heat bath on faces: an interior face whose four edge neighbours
 * share the height m is resampled to m+1 or m-1 with the conditional
 * probability of the weights (its four corner vertices, which also see its
 * four diagonal neighbours).  Faces are coloured by (i mod 2, j mod 2); colour
 * step s of an epoch updates class s mod 4 (row parity (s mod 4) / 2, column
 * parity s mod 2), so a sweep is four colour steps, and each step draws one
 * 23-bit number per face from Philox4x32-10: faces (i, 8q + p + 2b), b = 0..3,
 * take output word b of counter (i Q + q, s lo, s hi, chain) under the epoch
 * key, Q = ceil((n+1)/8); up iff draw < the threshold of the face's diagonal
 * pattern.  Uniform weights sample alternating-sign matrices uniformly.
 */
#ifndef RT_B200_SIXV_H
#define RT_B200_SIXV_H

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rt_sixv rt_sixv;

/* A handle on one device (its own stream); weights start uniform. */
rt_status rt_sixv_create(int32_t device, rt_sixv** out);
rt_status rt_sixv_destroy(rt_sixv* h);
const char* rt_sixv_last_error(rt_sixv* h);

/* Weights of the six vertex types a1, a2, b1, b2, c1, c2 (finite, > 0). */
rt_status rt_sixv_set_weights(rt_sixv* h, const double w[6]);

/* The 16 integer thresholds of the heat bath under the current weights:
 * entry p (bit 0 NW, 1 NE, 2 SW, 3 SE diagonal neighbour at m+1) is
 * ceil(P(up) 2^23).  *monotone = 1 when raising any diagonal neighbour never
 * lowers P(up) -- the condition under which rt_sixv_cftp is exact. */
rt_status rt_sixv_thresholds(rt_sixv* h, uint32_t thr[16], int32_t* monotone);

/* Minimal (|i-j|) and maximal (min(i+j, 2n-i-j)) domain-wall height
 * functions, (n+1)^2 each; either pointer may be NULL. */
rt_status rt_sixv_dwbc_heights(int32_t n, int32_t* hmin, int32_t* hmax);

/* RT_OK when h is a domain-wall height function of the n x n grid. */
rt_status rt_sixv_check(const int32_t* heights, int32_t n);

/* The alternating-sign matrix (n x n, entries -1, 0, 1) and the vertex
 * types (n x n, 0..5) of a valid height function. */
rt_status rt_sixv_to_asm(const int32_t* heights, int32_t n, int32_t* asm_out);
rt_status rt_sixv_vertex_types(const int32_t* heights, int32_t n, int32_t* types);

/* `sweeps` sweeps of the heat bath on the host heights ((n+1)^2, updated in
 * place; n <= 32000), epoch key `key`, Philox counter word 3 `chain`.
 * Synchronous.  At most 2^38 sweeps; more is RT_E_INVAL. */
rt_status rt_sixv_walk(rt_sixv* h, int32_t* heights, int32_t n, int64_t sweeps, uint64_t key, uint32_t chain);

/* Coupling from the past (no reference counterpart beyond the domino driver
 * Examples/AztecDiamondCftpEx.cpp:42-68, whose pattern it follows): chains
 * from the maximal and minimal heights run as two lattices of one launch
 * through the same epochs, newest first, keyed by successive
 * std::mt19937(master_seed) outputs; the schedule doubles from first_sweeps
 * until they agree.  Exact when the weights are monotone (see
 * rt_sixv_thresholds), else RT_E_INVAL.  out_heights (optional) receives the
 * sample; stats counts colour steps (four per sweep).  A schedule that
 * would pass 2^38 sweeps in one trial ends with RT_E_INVAL. */
rt_status rt_sixv_cftp(rt_sixv* h, int32_t n, int64_t first_sweeps, int64_t master_seed, int32_t max_trials,
                       int32_t* out_heights, rt_cftp_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_SIXV_H */
