"""The height projection's CPU restatement (oracle/rt_oracle.c,
orc_project_heights): valid height functions between the extremal ones,
exact on valid inputs, and the tilings they give match the reference's own
HeightfuncToTiling where oracle/_ref is built."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po
from projection_check import INF, check_height_function


def _domain(model: str, size: int):
    import randomtilings_b200 as rt

    if model == "domino":
        return rt.DominoTiler.AztecDiamond(size)
    return rt.LozengeTiler.Hexagon(size, size + 2, max(1, size - 1))


def _targets(hmin, hmax, seed):
    rng = np.random.default_rng(seed)
    lo, hi = hmin.astype(np.float64), hmax.astype(np.float64)
    inside = hmin != INF
    mid = np.where(inside, (lo + hi) / 2, 0)
    noise = rng.normal(0, 3, size=hmin.shape)
    yield np.where(inside, mid, 0).astype(np.float32)                     # smooth middle surface
    yield np.where(inside, mid + noise, 0).astype(np.float32)             # noisy
    yield np.where(inside, lo + rng.uniform(-5, 5, hmin.shape) * 4, 0).astype(np.float32)
    yield np.where(inside, rng.uniform(lo.min() - 10, hi.max() + 10, hmin.shape), 0).astype(np.float32)


@pytest.mark.parametrize("model,size", [("domino", 5), ("domino", 12), ("lozenge", 3), ("lozenge", 7)])
def test_projection_is_a_valid_height_function(model, size):
    from randomtilings_b200.project import extremal_heights

    import randomtilings_b200 as rt

    code = rt.RT_DOMINO if model == "domino" else rt.RT_LOZENGE
    d = _domain(model, size)
    hmin, hmax = extremal_heights(code, d)
    for k, t in enumerate(_targets(hmin, hmax, size)):
        h = po.project_heights(model, d, hmin, hmax, t)
        check_height_function(model, d, h, hmin, hmax)


@pytest.mark.parametrize("model,size", [("domino", 9), ("lozenge", 6)])
def test_projection_keeps_valid_heights(model, size):
    """A valid height function (of a random tiling) projects onto itself, and
    the extremal ones onto themselves."""
    import randomtilings_b200 as rt
    from randomtilings_b200.project import extremal_heights

    code = rt.RT_DOMINO if model == "domino" else rt.RT_LOZENGE
    cls = rt.DominoTiler if model == "domino" else rt.LozengeTiler
    d = _domain(model, size)
    hmin, hmax = extremal_heights(code, d)
    t = po.walk_fast("domino" if model == "domino" else "lozenge", cls.MinTiling(d), 500, 3)
    h = np.asarray(cls.TilingToHeightfunc(t, d), dtype=np.int32)
    for valid in (h, hmin, hmax):
        assert np.array_equal(po.project_heights(model, d, hmin, hmax, valid.astype(np.float32)), valid)
    big = np.where(hmin != INF, 1e6, 0).astype(np.float32)
    assert np.array_equal(po.project_heights(model, d, hmin, hmax, big), hmax)
    assert np.array_equal(po.project_heights(model, d, hmin, hmax, -big), hmin)


@pytest.mark.skipif(not po.have_ref(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("model,size", [("domino", 8), ("lozenge", 5)])
def test_projected_tiling_equals_reference_heightfunc_to_tiling(model, size):
    import randomtilings_b200 as rt
    from randomtilings_b200.project import extremal_heights

    code = rt.RT_DOMINO if model == "domino" else rt.RT_LOZENGE
    cls = rt.DominoTiler if model == "domino" else rt.LozengeTiler
    d = _domain(model, size)
    hmin, hmax = extremal_heights(code, d)
    for t in _targets(hmin, hmax, 7):
        h = po.project_heights(model, d, hmin, hmax, t)
        ref = po.ref_build(f"{model}_h2t", h, d)
        assert np.array_equal(np.asarray(cls.HeightfuncToTiling(h, d)), ref)
