"""The compact binary matrix format (rt_save_matrix_binary /
rt_load_matrix_binary): exact round trips of tilings, heights and domains,
the width it picks, and refusal of files that are not intact.  No GPU."""
from __future__ import annotations

import os

import numpy as np
import pytest

import randomtilings_b200 as rt
from randomtilings_b200 import _capi, builders

HEADER = 40


def _arrays():
    D, L = rt.DominoTiler, rt.LozengeTiler
    az = D.AztecDiamond(40)
    hx = L.AlmostHexDomain(30, 2)
    t = np.asarray(D.MinTiling(az))
    return {
        "domino_tiling": (t, 4),
        "domino_domain": (np.asarray(az), 1),
        "lozenge_tiling": (np.asarray(L.MaxTiling(hx)), 8),
        "domino_heights": (np.asarray(D.TilingToHeightfunc(t, az)), 32),  # INT_MAX outside the domain
        "tridimer_tiling": (np.asarray(rt.TriangleDimerTiler.IceCreamCone(20, 3)), 4),
        "recttri_tiling": (np.asarray(rt.RectTriangleTiler.maxHex(12)), 32),  # six hex digits per vertex
        "negative_small": (np.array([-3, -1, 0, 2, 4], dtype=np.int32), 4),
        "constant": (np.full(1000, 7, dtype=np.int32), 1),
        "one": (np.array([123456], dtype=np.int32), 1),
        "extremes": (np.array([np.iinfo(np.int32).min, 0, np.iinfo(np.int32).max], dtype=np.int32), 32),
        "wide": (np.arange(70000, dtype=np.int32) * 3 - 5, 32),
        "sixteen": (np.arange(40000, dtype=np.int32), 16),
    }


@pytest.mark.parametrize("name", sorted(_arrays()))
def test_round_trip_and_width(name, tmp_path):
    a, bits = _arrays()[name]
    p = tmp_path / "m.bin"
    builders.save_matrix_binary(a, p)
    b = builders.load_matrix_binary(p)
    assert b.dtype == np.int32 and np.array_equal(b, a.reshape(-1))
    assert os.path.getsize(p) == HEADER + (a.size * bits + 7) // 8


def test_tiler_names(tmp_path):
    D = rt.DominoTiler
    t = np.asarray(D.MaxTiling(D.AztecDiamond(9)))
    D.SaveMatrixBinary(t, tmp_path / "t.bin")
    assert np.array_equal(D.LoadMatrixBinary(tmp_path / "t.bin"), t)


def test_empty_array(tmp_path):
    p = tmp_path / "e.bin"
    builders.save_matrix_binary(np.zeros(0, np.int32), p)
    assert builders.load_matrix_binary(p).size == 0


@pytest.mark.parametrize("damage", ["flip", "truncate", "extend", "magic", "bits"])
def test_damaged_files_are_refused(damage, tmp_path):
    a = np.asarray(rt.DominoTiler.MinTiling(rt.DominoTiler.AztecDiamond(12)))
    p = tmp_path / "m.bin"
    builders.save_matrix_binary(a, p)
    raw = bytearray(open(p, "rb").read())
    if damage == "flip":
        raw[HEADER + 17] ^= 0x10
    elif damage == "truncate":
        raw = raw[:-1]
    elif damage == "extend":
        raw += b"\0"
    elif damage == "magic":
        raw[0] = ord("X")
    else:
        raw[16] = 3
    open(p, "wb").write(bytes(raw))
    with pytest.raises(_capi.RtError):
        builders.load_matrix_binary(p)


def test_text_file_is_not_binary(tmp_path):
    p = tmp_path / "m.txt"
    builders.save_matrix(np.arange(16, dtype=np.int32), p)
    with pytest.raises(_capi.RtError):
        builders.load_matrix_binary(p)


@pytest.mark.parametrize("count,bits", [(1 << 40, 32), ((1 << 40) - 1, 1), (1 << 33, 8), (5, 32)])
def test_header_that_overstates_the_payload_is_refused(count, bits, tmp_path):
    """A header announcing more values than the file holds is refused from the
    file's size, before a buffer is sized from the header: a count of 2^40
    32-bit values must not become a 4 TB allocation."""
    p = tmp_path / "forged.bin"
    head = bytearray(HEADER)
    head[:8] = b"RTBMAT1\0"
    head[8:16] = count.to_bytes(8, "little")
    head[16:20] = bits.to_bytes(4, "little")
    open(p, "wb").write(bytes(head) + b"\0" * 16)
    lib = _capi.load()
    import ctypes

    n = ctypes.c_int64(-1)
    assert lib.rt_load_matrix_binary(str(p).encode(), None, 0, ctypes.byref(n)) == _capi.RT_E_INVAL
    assert n.value == -1
