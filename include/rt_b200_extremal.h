/* rt_b200_extremal.h -- the extremal tilings of a domino or lozenge domain
 * and their height functions, computed on the GPU.
 *
 * Replaces, for large domains, DominoTiler::MaxTiling / MinTiling
 * (src/Domino/DominoTiler.cpp:214-399), LozengeTiler::MinTiling / MaxTiling
 * (src/Lozenge/LozengeTiler.cpp:140-318) and the TilingToHeightfunc of their
 * results (DominoTiler.cpp:423-461, LozengeTiler.cpp:95-138).  The results
 * are the same arrays as those host functions return (and as
 * rt_domino_max_tiling ... in rt_b200_host.h): tilings in the reference's
 * vertex-bit encoding, heights 0 at the first boundary vertex in row-major
 * order and INT_MAX outside the domain.
 *
 * Method (Thurston's construction, as the reference): the heights of the
 * boundary are fixed by a walk along the boundary edges (host, only the
 * boundary vertices are visited); the maximal height function is then the
 * smallest reach of the boundary along height-increasing edges, h(w) =
 * min over in-neighbours v of h(v) + 1, and the minimal one the mirror
 * image.  The reference floods breadth-first on the host; here both
 * functions are relaxed together to that fixpoint, 32 x 64-vertex tiles at a
 * time in shared memory, passes repeating over the tiles whose halo changed
 * until one pass changes nothing.  The tilings follow from the height
 * differences (HeightfuncToTiling, DominoTiler.cpp:402-421,
 * LozengeTiler.cpp:321-342).  A domain whose boundary heights disagree or
 * whose flood overruns a boundary height is not tileable (RT_E_INVAL, as the
 * host functions).
 */
#ifndef RT_B200_EXTREMAL_H
#define RT_B200_EXTREMAL_H

#include "rt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t n;            /* vertex side: every output is n x n */
    int64_t boundary;     /* boundary vertices fixed by the walk */
    int64_t passes;       /* relaxation passes over the tiles */
    int64_t tile_updates; /* tiles that changed, summed over the passes */
    double device_ms;     /* device time from the uploaded domain to the finished outputs */
    double walk_ms;       /* host: the boundary walk */
    double alloc_ms;      /* host: device allocations */
    double upload_ms;     /* host: copy of the domain and the boundary heights to the device */
    double download_ms;   /* host: copies of the requested outputs back */
} rt_extremal_stats;

/* model: RT_DOMINO or RT_LOZENGE.  d, dlen: the domain as the builders
 * return it (AztecDiamond, AlmostHexDomain, rt_lozenge_hexagon ...).  Each of
 * tmin, tmax, hmin, hmax is NULL or a host array of len = n*n int32
 * (n = sqrt(dlen) + 1 for dominoes, sqrt(dlen / 2) + 1 for lozenges);
 * tmin / hmin receive MinTiling and its height function, tmax / hmax
 * MaxTiling and its.  Synchronous; runs on `device`. */
rt_status rt_extremal_tilings(int32_t model, const int32_t* d, int64_t dlen, int32_t device, int32_t* tmin,
                              int32_t* tmax, int32_t* hmin, int32_t* hmax, int64_t len, rt_extremal_stats* stats);

/* The same results written into the caller's device buffers (each NULL or
 * n*n int32 of device memory on `device`, which also serve as the working
 * arrays): no copy back to the host, for callers that go on on the GPU
 * (e.g. rt_walk_device_noalloc from d_tmin).  Outputs that are not device
 * memory of `device` are rejected with RT_E_INVAL before anything runs.
 * Synchronous; the stats' download_ms is then only the final wait. */
rt_status rt_extremal_tilings_device(int32_t model, const int32_t* d, int64_t dlen, int32_t device, int32_t* d_tmin,
                                     int32_t* d_tmax, int32_t* d_hmin, int32_t* d_hmax, int64_t len,
                                     rt_extremal_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_EXTREMAL_H */
