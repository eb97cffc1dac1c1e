/* rt_b200_project.h -- exact projection of a real-valued height surface onto
 * the height function of a tiling (dominoes, lozenges).
 *
 * No reference counterpart; it feeds the reference's HeightfuncToTiling
 * (src/Domino/DominoTiler.cpp:402-461, src/Lozenge/LozengeTiler.cpp:95-138,
 * rt_domino_height_to_tiling / rt_lozenge_height_to_tiling here).  Heights
 * live on the tiling's N x N vertices in the reference's normalisation
 * (0 at the first boundary vertex, INT_MAX outside the domain).  A valid
 * height function h has h(v) = h_min(v) mod M (M = 4 for dominoes, 3 for
 * lozenges) and, along every edge v -> w that touches the domain, changes by
 * s or by -(M-1)s, where s = +-1 is the edge's orientation step; equivalently
 * h(w) - h(v) <= 1 where s = +1 and <= M-1 where s = -1.
 *
 * Steps (exact integer arithmetic after the first):
 *   1. residue rounding: g(v) = h_min(v) + M * floor((t(v) - h_min(v)) / M + 1/2)
 *      (in double precision), clamped to [h_min(v), h_max(v)]; boundary
 *      vertices take h_min(v) (= h_max(v));
 *   2. min-plus relaxation to the largest g' <= g that satisfies every edge
 *      constraint into an interior vertex (boundary vertices stay fixed);
 *   3. h = max(g', h_min) pointwise.
 * The result is a valid height function with h_min <= h <= h_max, equal to
 * the input wherever the input already was one.
 */
#ifndef RT_B200_PROJECT_H
#define RT_B200_PROJECT_H

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t passes;     /* relaxation passes until no vertex changed */
    int64_t lowered;    /* vertices step 2 lowered */
    int64_t raised;     /* vertices step 3 raised back to h_min */
    double device_ms;   /* device time of steps 1-3 */
} rt_project_stats;

/* model: RT_DOMINO or RT_LOZENGE.  d: the domain (as AztecDiamond /
 * AlmostHexDomain return it); hmin, hmax: the height functions of the
 * minimal and maximal tilings (TilingToHeightfunc); target: n*n floats
 * (ignored outside the domain); out: n*n int32.  Runs on `device`. */
rt_status rt_project_heights(int32_t model, const int32_t* d, int64_t dlen, const int32_t* hmin,
                             const int32_t* hmax, const float* target, int32_t* out, int64_t hlen, int32_t device,
                             rt_project_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_PROJECT_H */
