/* rt_b200_height.h -- height functions of device-resident tilings
 * (dominoes, lozenges): the statistics kernels of the learned warm start and
 * of the warm / cold comparison.
 *
 * Replaces, on the device, DominoTiler::TilingToHeightfunc
 * (src/Domino/DominoTiler.cpp:423-461) and LozengeTiler::TilingToHeightfunc
 * (src/Lozenge/LozengeTiler.cpp:95-138), which walk the tiling breadth-first
 * on the host.  The result is the same array: 0 at the first boundary vertex
 * in row-major order, INT_MAX outside the domain.
 *
 * Method.  Along an edge that touches the domain the height changes by the
 * edge's orientation step s (+-1) when no tile crosses it and by -3s
 * (dominoes) or -2s (lozenges) when one does, so the height of a row is a
 * prefix sum of per-edge steps, and consecutive rows are tied together by
 * one vertical edge each.  A plan, built once per domain on the host,
 * records each vertex row's run [lo, hi] of domain vertices and the column of
 * the edge tying it to the row above.  It accepts domains whose every vertex
 * row is one run of domain vertices joined by in-domain edges, with
 * consecutive non-empty rows (Aztec diamonds, a x b x c hexagons and the
 * reference's AlmostHexDomain among them); others are rejected with
 * RT_E_INVAL at plan creation, and the host functions in rt_b200_host.h
 * remain for them.
 *
 * All pointers named d_* are device memory (the device the plan was created
 * on); calls are asynchronous on `stream` (a cudaStream_t, NULL = the legacy
 * default stream) unless stated otherwise.  A plan owns n*n*4 + O(n) bytes of
 * device scratch; one plan is not safe to use from two host threads at once.
 */
#ifndef RT_B200_HEIGHT_H
#define RT_B200_HEIGHT_H

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rt_hplan rt_hplan;

/* model: RT_DOMINO or RT_LOZENGE; d: the domain as the builders return it
 * (AztecDiamond, AlmostHexDomain, rt_lozenge_hexagon ...). */
rt_status rt_hplan_create(int32_t model, const int32_t* d, int64_t dlen, int32_t device, rt_hplan** out);
rt_status rt_hplan_destroy(rt_hplan* p);
/* Vertex side n (tilings and heights are n x n) and number of domain vertices. */
rt_status rt_hplan_info(rt_hplan* p, int32_t* n, int64_t* vertices);
const char* rt_hplan_last_error(rt_hplan* p);

/* Heights of the n x n device tiling d_tiling into d_heights (n x n int32). */
rt_status rt_hplan_heights(rt_hplan* p, const int32_t* d_tiling, int32_t* d_heights, void* stream);
/* d_sum[v] += h(v) at every domain vertex (n x n int64); other entries untouched.
 * Mean height surfaces are sums over samples divided by their count. */
rt_status rt_hplan_accumulate(rt_hplan* p, const int32_t* d_tiling, int64_t* d_sum, void* stream);
/* Mean over domain vertices of |h(v) - d_ref[v]| (d_ref: n x n float).
 * Synchronous: waits for the stream and writes *mean_abs on the host. */
rt_status rt_hplan_error(rt_hplan* p, const int32_t* d_tiling, const float* d_ref, double* mean_abs, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_HEIGHT_H */
