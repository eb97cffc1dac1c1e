"""Large pictures, where the writers format blocks of rows on several
threads: the same bytes whatever the thread count, and the same bytes as the
reference's own writers (oracle/_ref, when it is built) on domains far larger
than the golden cases.  No GPU needed."""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

import randomtilings_b200 as rt
from oracle import pyoracle as po


def _sha(path) -> str:
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def _cases():
    D, L, T = rt.DominoTiler, rt.LozengeTiler, rt.TriangleDimerTiler
    # sizes well above the 65,536 cells from which rows are formatted on several threads
    az = D.AztecDiamond(150)
    hx = L.AlmostHexDomain(160, 3)
    out = [("domino_tiling", "rt_domino_tiling_svg", D.MinTiling(az), None),
           ("domino_dimer_d", "rt_domino_dimer_svg", D.MaxTiling(az), az),
           ("domino_dimer", "rt_domino_dimer_svg", D.MinTiling(az), None),
           ("lozenge_tiling", "rt_lozenge_tiling_svg", L.MaxTiling(hx), None),
           ("lozenge_dimer_d", "rt_lozenge_dimer_svg", L.MinTiling(hx), hx),
           ("lozenge_domain", "rt_lozenge_domain_svg", hx, None),
           ("save_matrix", "rt_save_matrix", L.MinTiling(hx), None),
           ("tridimer_tiling", "rt_tridimer_tiling_svg", T.IceCreamCone(270, 4), None),
           ("recttri_tiling", "rt_recttri_tiling_svg", rt.RectTriangleTiler.maxHex(48), None)]
    return out


@pytest.mark.skipif(not po.have_ref(), reason="oracle/_ref (the reference built from its sources) is absent")
@pytest.mark.parametrize("k", range(9))
def test_large_pictures_equal_the_reference(k, tmp_path):
    cases = _cases()
    if k >= len(cases):
        pytest.skip("no such case")
    ref_name, fn, a, b = cases[k]
    ours, theirs = tmp_path / "ours", tmp_path / "ref"
    rt.builders.write(fn, str(ours), *([a, b] if "dimer_svg" in fn else [a]))
    po.ref_write(ref_name, str(theirs), a, b)
    assert np.asarray(a).size * (8 if "recttri" in fn else 1) >= 1 << 16  # (a face is drawn as ~8 cells)
    assert _sha(ours) == _sha(theirs)


def test_thread_count_does_not_change_the_bytes(tmp_path):
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import randomtilings_b200 as rt\n"
        "D = rt.DominoTiler; d = D.AztecDiamond(120)\n"
        "D.DimerToSVG(D.MinTiling(d), d, sys.argv[1])\n"
        "rt.LozengeTiler.TilingToSVG(rt.LozengeTiler.MaxTiling(rt.LozengeTiler.AlmostHexDomain(90, 0)), sys.argv[2])\n"
    ) % ROOT
    digests = set()
    for th in ("1", "2", "7"):
        p1, p2 = tmp_path / f"a{th}", tmp_path / f"b{th}"
        subprocess.run([sys.executable, "-c", code, str(p1), str(p2)], check=True,
                       env=dict(os.environ, RT_WRITER_THREADS=th))
        digests.add((_sha(p1), _sha(p2)))
    assert len(digests) == 1
