"""ctypes binding of include/rt_b200.h (librt_b200.so).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

from . import _build

RT_OK = 0
RT_E_INVAL = -1
RT_E_PARAMS = -2
RT_E_NOMEM = -3
RT_E_CUDA = -4
RT_E_TIMEOUT = -5
RT_E_NODEVICE = -6
RT_E_STATE = -7

RT_DOMINO, RT_LOZENGE, RT_RECTTRI, RT_TRIDIMER = 0, 1, 2, 3
RT_KERNEL_DEFAULT, RT_KERNEL_CFTP, RT_KERNEL_QWEIGHT = 0, 1, 2
RT_RNG_TINYMT, RT_RNG_PHILOX, RT_RNG_PLANES = 0, 1, 2
RT_QCMP_FLOAT32, RT_QCMP_DOUBLE = 0, 1

_STATUS_NAMES = {
    RT_OK: "RT_OK", RT_E_INVAL: "RT_E_INVAL", RT_E_PARAMS: "RT_E_PARAMS", RT_E_NOMEM: "RT_E_NOMEM",
    RT_E_CUDA: "RT_E_CUDA", RT_E_TIMEOUT: "RT_E_TIMEOUT", RT_E_NODEVICE: "RT_E_NODEVICE",
    RT_E_STATE: "RT_E_STATE",
}


class RtError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")


class RtConfig(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int32),
        ("kernel", ctypes.c_int32),
        ("rng", ctypes.c_int32),
        ("qcmp", ctypes.c_int32),
        ("q", ctypes.c_double),
        ("weights", ctypes.c_float * 16),
        ("device", ctypes.c_int32),
        ("chain", ctypes.c_uint32),
        ("stream", ctypes.c_void_p),
    ]


class RtCftpStats(ctypes.Structure):
    _fields_ = [
        ("total_steps", ctypes.c_int64),
        ("trials", ctypes.c_int32),
        ("coalesced", ctypes.c_int32),
        ("device_ms", ctypes.c_double),
    ]


RT_CFTP_DOUBLING, RT_CFTP_REFERENCE = 0, 1


class RtChain(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int32),
        ("kernel", ctypes.c_int32),
        ("chain", ctypes.c_uint32),
        ("q", ctypes.c_float),
        ("key", ctypes.c_int64),
    ]


class RtBatchInfo(ctypes.Structure):
    _fields_ = [
        ("chains", ctypes.c_int32),
        ("cluster", ctypes.c_int32 * 6),
        ("block", ctypes.c_int32 * 6),
        ("clusters", ctypes.c_int32 * 6),
        ("tune_ms", ctypes.c_double),
        ("run_ms", ctypes.c_double),
        ("attempts", ctypes.c_int64),
        ("algorithmic_bytes", ctypes.c_int64),
        ("sweeps_per_launch", ctypes.c_int64 * 6),
    ]

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64

# name -> (restype, argtypes); every symbol the header declares.
SIGNATURES = {
    "rt_config_default": (None, [ctypes.POINTER(RtConfig), _I32]),
    "rt_create": (ctypes.c_int, [ctypes.POINTER(RtConfig), ctypes.POINTER(_P)]),
    "rt_destroy": (ctypes.c_int, [_P]),
    "rt_load_rng_params": (ctypes.c_int, [_P, ctypes.c_char_p, _I64]),
    "rt_set_rng_params": (ctypes.c_int, [_P, _P, _I64]),
    "rt_set_domino_weights": (ctypes.c_int, [_P, _I32, _P, _P]),
    "rt_set_lozenge_weights": (ctypes.c_int, [_P, _I32, _P, _P, _P]),
    "rt_walk": (ctypes.c_int, [_P, _P, _I32, _I64, _I64]),
    "rt_walk_epochs": (ctypes.c_int, [_P, _P, _I32, _P, _P, _I32]),
    "rt_cftp": (ctypes.c_int, [_P, _P, _P, _I32, _I64, _I32, _I64, _I32, _P, ctypes.POINTER(RtCftpStats)]),
    "rt_upload": (ctypes.c_int, [_P, _P, _I32]),
    "rt_run": (ctypes.c_int, [_P, _I64, _I64]),
    "rt_download": (ctypes.c_int, [_P, _P]),
    "rt_synchronize": (ctypes.c_int, [_P]),
    "rt_stream": (_P, [_P]),
    "rt_device_tiling": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "rt_last_run_info": (ctypes.c_int, [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    "rt_last_error": (ctypes.c_char_p, [_P]),
    "rt_version": (ctypes.c_char_p, []),
    "rt_walk_device_noalloc": (ctypes.c_int, [ctypes.POINTER(RtConfig), _P, _I32, _I64, _I64,
                                              ctypes.POINTER(ctypes.c_char), ctypes.c_size_t]),
}

_PL = ctypes.POINTER(_I64)
# include/rt_b200_host.h: every builder writes (out, cap) and reports *len.
HOST_SIGNATURES = {
    "rt_domino_rectangle": [_I32, _I32],
    "rt_domino_aztec_rectangle": [_I32, _P, _I32],
    "rt_domino_aztec": [_I32],
    "rt_domino_domain_to_vertices": [_P, _I64],
    "rt_domino_max_tiling": [_P, _I64],
    "rt_domino_min_tiling": [_P, _I64],
    "rt_domino_height_to_tiling": [_P, _I64, _P, _I64],
    "rt_domino_tiling_to_height": [_P, _I64, _P, _I64],
    "rt_domino_tiling_to_domain": [_P, _I64],
    "rt_lozenge_almost_hex": [_I32, _I32],
    "rt_lozenge_hexagon": [_I32, _I32, _I32],
    "rt_lozenge_domain_to_vertices": [_P, _I64],
    "rt_lozenge_max_tiling": [_P, _I64],
    "rt_lozenge_min_tiling": [_P, _I64],
    "rt_lozenge_height_to_tiling": [_P, _I64, _P, _I64],
    "rt_lozenge_tiling_to_height": [_P, _I64, _P, _I64],
    "rt_lozenge_tiling_to_domain": [_P, _I64],
    "rt_recttri_max_hex": [_I32],
    "rt_recttri_min_hex": [_I32],
    "rt_recttri_from_lozenge": [_P, _I64, _P, _I64],
    "rt_tridimer_ice_cream_cone": [_I32, _I32],
    "rt_tridimer_test_butterfly": [_I32],
    "rt_tridimer_hexagon": [_I32],
    "rt_tridimer_triangle_flips": [_P, _I64],
    "rt_tridimer_butterfly_flips": [_P, _I64],
    "rt_tridimer_vertices": [_P, _I64],
    "rt_tridimer_tiling_to_domain": [_P, _I64],
    "rt_tridimer_dimer_indicator": [_P, _I64, _I32],
}
for _name, _args in HOST_SIGNATURES.items():
    SIGNATURES[_name] = (ctypes.c_int, [*_args, _P, _I64, _PL])

_S = ctypes.c_char_p
# include/rt_b200_svg.h
SIGNATURES.update({
    "rt_domino_domain_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_domino_tiling_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_domino_maya_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_domino_dimer_svg": (ctypes.c_int, [_P, _I64, _P, _I64, _S]),
    "rt_lozenge_domain_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_lozenge_tiling_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_lozenge_dimer_svg": (ctypes.c_int, [_P, _I64, _P, _I64, _S]),
    "rt_lozenge_print_domain": (ctypes.c_int, [_P, _I64, _S]),
    "rt_recttri_tiling_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_tridimer_domain_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_tridimer_tiling_svg": (ctypes.c_int, [_P, _I64, _S]),
    "rt_tridimer_dimer_svg": (ctypes.c_int, [_P, _I64, _P, _I64, _S]),
    "rt_save_matrix": (ctypes.c_int, [_P, _I64, _S]),
    "rt_load_matrix": (ctypes.c_int, [_S, _P, _I64, _PL]),
    "rt_save_matrix_binary": (ctypes.c_int, [_P, _I64, _S]),
    "rt_load_matrix_binary": (ctypes.c_int, [_S, _P, _I64, _PL]),
})

# include/rt_b200_batch.h
SIGNATURES.update({
    "rt_batch_create": (ctypes.c_int, [_I32, ctypes.POINTER(_P)]),
    "rt_batch_destroy": (ctypes.c_int, [_P]),
    "rt_batch_add": (ctypes.c_int, [_P, ctypes.POINTER(RtChain), _P, _I32, _PL]),
    "rt_batch_set_tuning": (ctypes.c_int, [_P, _I32, _I32, _I32]),
    "rt_batch_run": (ctypes.c_int, [_P, _I64]),
    "rt_batch_set_sweeps_per_launch": (ctypes.c_int, [_P, _I64]),
    "rt_batch_download": (ctypes.c_int, [_P, _I64, _P]),
    "rt_batch_device_tiling": (ctypes.c_int, [_P, _I64, _P, _P]),
    "rt_batch_get_info": (ctypes.c_int, [_P, ctypes.POINTER(RtBatchInfo)]),
    "rt_batch_last_error": (ctypes.c_char_p, [_P]),
    "rt_mixed_chain_spec": (ctypes.c_int, [_I64, ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
})


class RtProjectStats(ctypes.Structure):
    _fields_ = [("passes", ctypes.c_int64), ("lowered", ctypes.c_int64), ("raised", ctypes.c_int64),
                ("device_ms", ctypes.c_double)]


# include/rt_b200_project.h
SIGNATURES["rt_project_heights"] = (ctypes.c_int, [_I32, _P, _I64, _P, _P, _P, _P, _I64, _I32,
                                                   ctypes.POINTER(RtProjectStats)])



class RtExtremalStats(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("boundary", ctypes.c_int64), ("passes", ctypes.c_int64),
                ("tile_updates", ctypes.c_int64), ("device_ms", ctypes.c_double), ("walk_ms", ctypes.c_double),
                ("alloc_ms", ctypes.c_double), ("upload_ms", ctypes.c_double), ("download_ms", ctypes.c_double)]


# include/rt_b200_extremal.h
SIGNATURES["rt_extremal_tilings"] = (ctypes.c_int, [_I32, _P, _I64, _I32, _P, _P, _P, _P, _I64,
                                                    ctypes.POINTER(RtExtremalStats)])
SIGNATURES["rt_extremal_tilings_device"] = (ctypes.c_int, [_I32, _P, _I64, _I32, _P, _P, _P, _P, _I64,
                                                           ctypes.POINTER(RtExtremalStats)])

# include/rt_b200_height.h
SIGNATURES.update({
    "rt_hplan_create": (ctypes.c_int, [_I32, _P, _I64, _I32, ctypes.POINTER(_P)]),
    "rt_hplan_destroy": (ctypes.c_int, [_P]),
    "rt_hplan_info": (ctypes.c_int, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I64)]),
    "rt_hplan_last_error": (ctypes.c_char_p, [_P]),
    "rt_hplan_heights": (ctypes.c_int, [_P, _P, _P, _P]),
    "rt_hplan_accumulate": (ctypes.c_int, [_P, _P, _P, _P]),
    "rt_hplan_error": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_double), _P]),
})

# include/rt_b200_mlp.h
RT_MLP_IN, RT_MLP_WIDTH = 8, 128
RT_MLP_PARAMS = 128 * 8 + 128 + 128 * 128 + 128 + 128 * 128 + 128 + 128 + 1
SIGNATURES.update({
    "rt_mlp_create": (ctypes.c_int, [_I32, ctypes.c_uint64, ctypes.POINTER(_P)]),
    "rt_mlp_destroy": (ctypes.c_int, [_P]),
    "rt_mlp_get_params": (ctypes.c_int, [_P, _P]),
    "rt_mlp_set_params": (ctypes.c_int, [_P, _P]),
    "rt_mlp_predict": (ctypes.c_int, [_P, _P, _I64, _P]),
    "rt_mlp_loss_grad": (ctypes.c_int, [_P, _P, _P, _I64, ctypes.POINTER(ctypes.c_float), _P]),
    "rt_mlp_set_data": (ctypes.c_int, [_P, _P, _P, _I64]),
    "rt_mlp_train": (ctypes.c_int, [_P, _I64, _I32, ctypes.c_float, ctypes.c_uint64,
                                    ctypes.POINTER(ctypes.c_float)]),
})

# include/rt_b200_sixv.h
SIGNATURES.update({
    "rt_sixv_create": (ctypes.c_int, [_I32, ctypes.POINTER(_P)]),
    "rt_sixv_destroy": (ctypes.c_int, [_P]),
    "rt_sixv_last_error": (ctypes.c_char_p, [_P]),
    "rt_sixv_set_weights": (ctypes.c_int, [_P, _P]),
    "rt_sixv_thresholds": (ctypes.c_int, [_P, _P, ctypes.POINTER(_I32)]),
    "rt_sixv_dwbc_heights": (ctypes.c_int, [_I32, _P, _P]),
    "rt_sixv_check": (ctypes.c_int, [_P, _I32]),
    "rt_sixv_to_asm": (ctypes.c_int, [_P, _I32, _P]),
    "rt_sixv_vertex_types": (ctypes.c_int, [_P, _I32, _P]),
    "rt_sixv_walk": (ctypes.c_int, [_P, _P, _I32, _I64, ctypes.c_uint64, ctypes.c_uint32]),
    "rt_sixv_cftp": (ctypes.c_int, [_P, _I32, _I64, _I64, _I32, _P, ctypes.POINTER(RtCftpStats)]),
})

_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Loads librt_b200.so (building it in-tree first if allowed)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise OSError(f"native library {path} is missing; run randomtilings_b200._build.build()")
        _build.build()
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, handle=None) -> None:
    if status != RT_OK:
        lib = load()
        msg = lib.rt_last_error(handle)
        raise RtError(status, msg.decode() if msg else "")
