"""Host-side checks of the bench-scale and float32 fixtures (no GPU).

* The library's host builders give the very start tilings whose walks
  tests/golden/bench_parity.json pins (the reference's MinTiling of the
  a=b=c=500 hexagon and of the Aztec diamond of order 2000).
* The oracle's C restatement agrees with the reference's q-lozenge kernel built
  in single precision (float32 comparison) and in double (qlozenge_f32.npz),
  and those fixtures do hold walks on which the two comparisons part.
* The Aztec n=100 walk (seed 42, 10,000 and 20,000 steps): the host
  TilingToHeightfunc of the reference's final tilings equals the
  reference's height functions.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, cases, golden
from oracle import pyoracle as po


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


@pytest.fixture(scope="module")
def want():
    with open(os.path.join(GOLDEN, "bench_parity.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


def test_hex500_start_matches_reference(rt, want):
    t = rt.LozengeTiler.MinTiling(rt.LozengeTiler.AlmostHexDomain(500, 0))
    assert digest(t) == want["hex500/start"]


def test_aztec2000_start_matches_reference(rt, want):
    t = rt.DominoTiler.MinTiling(rt.DominoTiler.AztecDiamond(2000))
    assert digest(t) == want["aztec2000/start"]


def test_hex500_fast_digest_is_the_restatement(rt, want):
    t = rt.LozengeTiler.MinTiling(rt.LozengeTiler.AlmostHexDomain(500, 0))
    assert digest(po.walk_fast("lozenge", t, 600, 42)) == want["hex500/fast/k42/600"]


@pytest.mark.parametrize("key", cases("qlozenge_f32", "qlozenge_f32/"))
def test_restatement_matches_float32_reference_build(key):
    g = golden("qlozenge_f32")
    t, steps, seed = g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0])
    assert np.array_equal(po.lozenge_walk(t, steps, seed, qweight=True, qcmp_double=False), g[f"{key}/end"])
    assert np.array_equal(po.lozenge_walk(t, steps, seed, qweight=True, qcmp_double=True), g[f"{key}/end_double"])


def test_float32_fixtures_exercise_the_divergence():
    g = golden("qlozenge_f32")
    parted = [k for k in cases("qlozenge_f32", "qlozenge_f32/hex40")
              if not np.array_equal(g[f"{k}/end"], g[f"{k}/end_double"])]
    assert len(parted) >= 3


@pytest.mark.parametrize("steps", [10000, 20000])
def test_aztec100_heights_on_host(rt, steps):
    b, c = golden("builders"), golden("aztec100")
    h = rt.DominoTiler.TilingToHeightfunc(c[f"cfg0/s{steps}/end"], b["domino/aztec100/domain"])
    assert np.array_equal(np.asarray(h), c[f"cfg0/s{steps}/height"])
