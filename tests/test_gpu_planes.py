"""Bit-plane mode (RT_RNG_PLANES): the bit-plane walk kernel equals the
oracle's per-site replay of the same rules and bits -- dominoes (toggle and
heat bath) and lozenges, one CTA and many (forced with RT_WALK_CTAS, so the
temporally blocked halo exchange runs at every depth RT_PLANE_DEPTH allows),
one and two lattices (CFTP), single walks and epochs."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


def _tiler(rt, model, kernel, ctas=0, depth=0, chain=0):
    os.environ["RT_WALK_CTAS"] = str(ctas)
    os.environ["RT_PLANE_DEPTH"] = str(depth)
    try:
        cls = rt.DominoTiler if model == "domino" else rt.LozengeTiler
        return cls(kernel=kernel, rng=rt.RT_RNG_PLANES, chain=chain)
    finally:
        os.environ.pop("RT_WALK_CTAS")
        os.environ.pop("RT_PLANE_DEPTH")


def _cases(rt):
    D, L = rt.DominoTiler, rt.LozengeTiler
    return [
        ("domino", 0, D.MinTiling(D.AztecDiamond(13))),
        ("domino", 1, D.MaxTiling(D.AztecDiamond(13))),
        ("domino", 0, D.MinTiling(D.AztecDiamond(70))),     # rows wider than one 128-site quad
        ("domino", 1, D.MinTiling(D.AztecDiamond(101))),    # odd order, ragged last word
        ("lozenge", 0, golden("builders")["lozenge/hex20_0/min"]),
        ("lozenge", 0, L.MinTiling(L.Hexagon(23, 40, 17))),
        ("lozenge", 0, L.MaxTiling(L.Hexagon(70, 50, 61))),
    ]


@pytest.mark.parametrize("k", range(7))
@pytest.mark.parametrize("ctas,depth", [(1, 0), (0, 0), (5, 1), (7, 3), (9, 0)])
def test_plane_walk_equals_oracle(rt, k, ctas, depth):
    model, kernel, t0 = _cases(rt)[k]
    name = "domino_cftp" if kernel == 1 else model
    steps, key = 61, 2**33 + 17 * k
    want = po.walk_planes(name, t0, steps, key, chain=3)
    tl = _tiler(rt, model, kernel, ctas, depth, chain=3)
    got = np.array(t0, dtype=np.int32)
    tl.Walk(got, steps, key)
    tl.close()
    assert not np.array_equal(got, np.asarray(t0)), "the walk changed nothing"
    assert np.array_equal(got, want)


@pytest.mark.parametrize("model,kernel", [("domino", 0), ("domino", 1), ("lozenge", 0)])
def test_plane_runs_compose_across_epochs(rt, model, kernel):
    """rt_walk_epochs / chained rt_run keys: epochs restart the step counter with their own key."""
    D, L = rt.DominoTiler, rt.LozengeTiler
    t0 = D.MinTiling(D.AztecDiamond(40)) if model == "domino" else L.MinTiling(L.Hexagon(30, 30, 30))
    name = "domino_cftp" if kernel == 1 else model
    want = po.walk_planes(name, po.walk_planes(name, t0, 30, 5), 43, 6)
    tl = _tiler(rt, model, kernel, 6, 0)
    tl.upload(t0)
    tl.run(30, 5)
    tl.run(43, 6)
    got = np.zeros(len(t0), dtype=np.int32)
    tl.download(got)
    tl.close()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("model", ["domino_cftp", "lozenge"])
@pytest.mark.parametrize("ctas", [0, 4])
def test_plane_cftp_equals_oracle(rt, model, ctas):
    D, L = rt.DominoTiler, rt.LozengeTiler
    if model == "domino_cftp":
        d = D.AztecDiamond(10)
        tmax, tmin, kernel, mm = D.MaxTiling(d), D.MinTiling(d), 1, "domino"
    else:
        d = L.Hexagon(6, 5, 7)
        tmax, tmin, kernel, mm = L.MaxTiling(d), L.MinTiling(d), 0, "lozenge"
    tl = _tiler(rt, mm, kernel, ctas, 0)
    got, st = tl.CFTP(tmax, tmin, first_steps=64, master_seed=9, max_trials=16)
    tl.close()
    want, trials, total, ok = po.cftp(tmax, tmin, 64, 9, max_trials=16, model=model, planes=True)
    assert st["coalesced"] and ok and st["trials"] == trials and st["total_steps"] == total
    assert np.array_equal(got, want)


def test_plane_mode_rejects_other_models(rt):
    with pytest.raises(rt.RtError):
        rt.RectTriangleTiler(rng=rt.RT_RNG_PLANES)
    with pytest.raises(rt.RtError):
        rt.LozengeTiler(kernel=rt.RT_KERNEL_QWEIGHT, rng=rt.RT_RNG_PLANES)


@pytest.mark.parametrize("model,kernel,ctas", [("domino", 0, 2), ("domino", 1, 3), ("lozenge", 0, 1)])
def test_plane_walk_four_words_per_item(rt, model, kernel, ctas):
    """Bands of more than 2048 words take four words (one Philox call) per work item."""
    D, L = rt.DominoTiler, rt.LozengeTiler
    t0 = D.MinTiling(D.AztecDiamond(300)) if model == "domino" else L.MinTiling(L.Hexagon(220, 200, 210))
    name = "domino_cftp" if kernel == 1 else model
    want = po.walk_planes(name, t0, 23, 99, chain=1)
    tl = _tiler(rt, model, kernel, ctas, 0, chain=1)
    got = np.array(t0, dtype=np.int32)
    tl.Walk(got, 23, 99)
    tl.close()
    assert np.array_equal(got, want)
