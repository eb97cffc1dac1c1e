// rt_tdops.h -- phase op codes of the triangle-dimer phase program
// (triangledimerkernel.cl's kernels, one op per array update), shared by the
// integer rule (rt_tridimer.cuh) and the bit-plane ops (rt_tdplane.cuh).
#pragma once

#include <stdint.h>

// The rule and the bit-plane ops compile for the device and, for the tests'
// host checks, for the host (where the including file declares WalkArgs and
// the phase-descriptor accessors the walk-kernel glue names).
#ifdef __CUDACC__
#define TD_HD __host__ __device__
#else
#define TD_HD inline
#endif

namespace rtb {

enum : uint32_t {
    TD_ROT_LOZ = 16,        // a = orientation t, b = class c           (RotateLozenges)            [draws]
    TD_LOZ_FLIPPED = 17,    // a = t, b = c                             (UpdateLozengesFlipped)
    TD_LOZ_OTHER = 18,      // a = t                                    (UpdateLozenges0/1/2)
    TD_UP_FROM_LOZ = 19,    //                                          (UpdateTriangleUFromLozenges)
    TD_TRI_OTHER = 20,      // a = 0: D from U, 1: U from D; b = butterflies refreshed from lozenges
    TD_ROT_TRI = 21,        // a = 1: down, 0: up; b = class c          (RotateTriangles)           [draws]
    TD_TRI_FLIPPED = 22,    // a = 1: down, 0: up; b = c                (UpdateTrianglesFlipped1/0)
    TD_LOZ_FROM_TRI = 23,   //                                          (UpdateLozenge{H,L,R}FromTriangles)
    TD_BFLY_FROM_LOZ = 24,  // b = butterfly mask; a = 1: also U from lozenges
    TD_ROT_BFLY = 25,       // a = t, b = p1 | p2 << 2                  (RotateButterflys)          [draws]
    TD_BFLY_SAME = 26,      // a = t, b = p1 | p2 << 2                  (UpdateButterflysFlipped?1)
    TD_BFLY_21 = 27,        // a = t, b = p1
    TD_BFLY_22 = 28,        // a = t, b = p1
    TD_BFLY_23_LOZ = 29     // a = t, b = p1: pass 23, then the lozenges from that butterfly array
};

}  // namespace rtb
