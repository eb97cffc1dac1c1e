"""B200-native (sm_100a) flip dynamics for random tilings.

The compute path is librt_b200.so (CUDA kernels behind the C ABI declared in
include/rt_b200.h); this package only binds it.  Importing the package does
not touch the GPU; creating a Tiler does.
"""
from ._capi import RtError, load  # noqa: F401
from .tilers import DominoTiler, LozengeTiler, RectTriangleTiler, TriangleDimerTiler  # noqa: F401

__all__ = ["DominoTiler", "LozengeTiler", "RectTriangleTiler", "TriangleDimerTiler", "RtError", "load"]
