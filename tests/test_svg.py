"""SVG and text writers of librt_b200.so: byte-identical to the reference's
(SHA-256 of the reference's own output on the same inputs, written by
tests/golden/make_golden.py), and to the reference's shipped example pictures
(Examples/ExampleOuts, digests in example_outputs.json).  No GPU needed."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

import randomtilings_b200 as rt

WRITERS = {
    "domino_domain": ("rt_domino_domain_svg", 1), "domino_tiling": ("rt_domino_tiling_svg", 1),
    "domino_maya": ("rt_domino_maya_svg", 1), "domino_dimer": ("rt_domino_dimer_svg", 2),
    "domino_dimer_d": ("rt_domino_dimer_svg", 2), "lozenge_domain": ("rt_lozenge_domain_svg", 1),
    "lozenge_tiling": ("rt_lozenge_tiling_svg", 1), "lozenge_dimer": ("rt_lozenge_dimer_svg", 2),
    "lozenge_dimer_d": ("rt_lozenge_dimer_svg", 2), "lozenge_print_domain": ("rt_lozenge_print_domain", 1),
    "recttri_tiling": ("rt_recttri_tiling_svg", 1), "tridimer_domain": ("rt_tridimer_domain_svg", 1),
    "tridimer_tiling": ("rt_tridimer_tiling_svg", 1), "tridimer_dimer": ("rt_tridimer_dimer_svg", 2),
    "tridimer_dimer_d": ("rt_tridimer_dimer_svg", 2), "save_matrix": ("rt_save_matrix", 1),
}

DIGESTS = json.load(open(os.path.join(GOLDEN, "svg_digests.json")))


def _get(key: str):
    return (golden("builders") if key[0] == "b" else golden("walks"))[key[2:]]


def _sha(path) -> str:
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


@pytest.mark.parametrize("case", sorted(DIGESTS))
def test_writer_matches_reference(case, tmp_path):
    parts = case.split(":")  # k : writer : src : key [: src : key | : None]
    writer, ka = parts[1], ":".join(parts[2:4])
    kb = None if parts[4] == "None" else ":".join(parts[4:6])
    fn, nargs = WRITERS[writer]
    arrays = [_get(ka)] + ([None if kb is None else _get(kb)] if nargs == 2 else [])
    out = tmp_path / "out"
    rt.builders.write(fn, out, *arrays)
    assert _sha(out) == DIGESTS[case]


EXAMPLES = json.load(open(os.path.join(GOLDEN, "example_outputs.json")))


def test_reference_example_pictures(tmp_path):
    """The reference's shipped pictures, regenerated from our builders + writers."""
    def check(name, fn, *arrays):
        path = tmp_path / name.replace("/", "_")
        fn(*arrays, str(path)) if arrays else fn(str(path))
        assert _sha(path) == EXAMPLES[name], name

    for n, name in ((5, "MaxTiling"), (5, "MinTiling")):
        t = getattr(rt.RectTriangleTiler, name[:3].lower() + "Hex")(n)
        check(f"RectTriangle/{name}.svg", rt.RectTriangleTiler.TilingToSVG, t)
        check(f"RectTriangle/{name}.txt", rt.RectTriangleTiler.SaveMatrix, t)
    d = rt.LozengeTiler.AlmostHexDomain(10, 2)
    check("MinimalLozenge/domainAlmostHex.svg", rt.LozengeTiler.DomainToSVG, d)
    check("MinimalLozenge/tilingStartAlmostHex.svg", rt.LozengeTiler.TilingToSVG, rt.LozengeTiler.MaxTiling(d))
    t = rt.TriangleDimerTiler.IceCreamCone(6, 0)
    dd = rt.TriangleDimerTiler.TilingToDomain(t)
    check("TriangleDimer/DimerStart.txt", rt.TriangleDimerTiler.SaveMatrix, t)
    check("TriangleDimer/Domain.txt", rt.TriangleDimerTiler.SaveMatrix, dd)
    check("TriangleDimer/Domain.svg", rt.TriangleDimerTiler.DomainToSVG, dd)
    check("TriangleDimer/TilingStart.svg", rt.TriangleDimerTiler.TilingToSVG, t)


def test_dimer_start_picture_differs_only_by_the_out_of_bounds_read(tmp_path):
    """TriangleDimerTiler::DimerToSVG (TriangleDimerTiler.cpp:876) reads the
    domain row above row 0, outside the vector.  The reference code built here
    and our writer both see an empty cell there; the picture the reference ships
    (Examples/ExampleOuts/TriangleDimer/DimerStart.svg) was written on a machine
    where that memory held a 1, which adds exactly one edge line in row 0.  The
    shipped file's digest (example_outputs.json) is that of our output plus that
    line, checked here through a stored copy of the one line."""
    t = rt.TriangleDimerTiler.IceCreamCone(6, 0)
    path = tmp_path / "dimer.svg"
    rt.TriangleDimerTiler.DimerToSVG(t, str(path))
    lines = open(path, "rb").read().split(b"\n")
    extra = b'<use xlink:href = "#eH" x = "3.5" y = "0"/>'
    patched = b"\n".join(lines[:12] + [extra] + lines[12:])
    assert hashlib.sha256(patched).hexdigest() == EXAMPLES["TriangleDimer/DimerStart.svg"]


def test_load_matrix_round_trip(tmp_path):
    t = golden("builders")["recttri/max_hex5"]
    p = tmp_path / "m.txt"
    rt.RectTriangleTiler.SaveMatrix(t, str(p))
    assert np.array_equal(rt.RectTriangleTiler.LoadMatrix(str(p)), t)


def test_load_matrix_long_digit_runs_wrap_like_the_reference(tmp_path):
    """LoadMatrix (common.cpp:141-161) reads every run of digits as one
    number ('-' and other characters only separate) into an int that wraps;
    runs of any length are read, keeping the value modulo 2^32 as int32."""
    from randomtilings_b200 import builders

    runs = ["7", "-12", "4294967297", "99999999999999999999999999", "2147483648", "0012"]
    p = tmp_path / "m.txt"
    p.write_text(" ".join(runs) + "\n")
    want = []
    for r in runs:
        v = int(r.lstrip("-")) % 2**32
        want.append(v - 2**32 if v >= 2**31 else v)
    assert builders.load_matrix(p).tolist() == want


def test_dimer_writers_on_inputs_the_builders_never_make(tmp_path):
    """A domino domain with cells in its last row (the reference's writer
    reads one row past the array there; the builders' padded domains never
    do), and triangle-dimer domains that do not belong to the tiling: a
    larger one is refused, and one whose length is not 2 m^2 is read only as
    far as its m x 2m cells."""
    import ctypes

    from randomtilings_b200 import _capi

    lib = _capi.load()
    path = str(tmp_path / "x.svg").encode()
    t = np.asarray(rt.DominoTiler.MaxTiling(rt.DominoTiler.AztecDiamond(3)), dtype=np.int32)
    m = int(round(t.size ** 0.5)) - 1
    d = np.ones(m * m, dtype=np.int32)
    assert lib.rt_domino_dimer_svg(t.ctypes.data, t.size, d.ctypes.data, d.size, path) == _capi.RT_OK

    tt = np.asarray(rt.TriangleDimerTiler.IceCreamCone(6, 1), dtype=np.int32)
    n = int(round(tt.size ** 0.5))
    big = np.ones(2 * (n // 2 + 1) ** 2, dtype=np.int32)
    assert lib.rt_tridimer_dimer_svg(tt.ctypes.data, tt.size, big.ctypes.data, big.size, path) == _capi.RT_E_INVAL
    ragged = np.ones(2 * (n // 2 + 1) ** 2 - 1, dtype=np.int32)  # the longest length that still reads as m = n / 2
    assert lib.rt_tridimer_dimer_svg(tt.ctypes.data, tt.size, ragged.ctypes.data, ragged.size, path) == _capi.RT_OK
