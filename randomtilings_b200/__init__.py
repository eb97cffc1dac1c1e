"""B200-native (sm_100a) flip dynamics for random tilings.

The compute path is librt_b200.so (CUDA kernels behind the C ABI declared in
include/rt_b200.h); this package only binds it.  Importing the package does
not touch the GPU; creating a Tiler does.
"""
from ._capi import (RT_CFTP_DOUBLING, RT_CFTP_REFERENCE, RT_DOMINO, RT_KERNEL_CFTP, RT_KERNEL_DEFAULT,  # noqa: F401
                    RT_KERNEL_QWEIGHT, RT_LOZENGE, RT_QCMP_DOUBLE, RT_QCMP_FLOAT32, RT_RECTTRI, RT_RNG_PHILOX, RT_RNG_PLANES,
                    RT_RNG_TINYMT, RT_TRIDIMER, RtError, load)
from .batch import Batch  # noqa: F401
from .sixvertex import SixVertexTiler  # noqa: F401
from .tilers import DominoTiler, LozengeTiler, RectTriangleTiler, TriangleDimerTiler  # noqa: F401

__all__ = ["DominoTiler", "LozengeTiler", "RectTriangleTiler", "TriangleDimerTiler", "SixVertexTiler", "Batch", "RtError", "load",
           "RT_KERNEL_DEFAULT", "RT_KERNEL_CFTP", "RT_KERNEL_QWEIGHT", "RT_RNG_TINYMT", "RT_RNG_PHILOX", "RT_RNG_PLANES",
           "RT_QCMP_FLOAT32", "RT_QCMP_DOUBLE", "RT_CFTP_DOUBLING", "RT_CFTP_REFERENCE", "RT_DOMINO", "RT_LOZENGE",
           "RT_RECTTRI", "RT_TRIDIMER"]
