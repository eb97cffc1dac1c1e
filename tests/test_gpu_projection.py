"""rt_project_heights on the GPU equals the oracle's projection (exact
integers) and yields valid height functions, up to Aztec order 300."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po
from projection_check import INF, check_height_function

pytestmark = pytest.mark.gpu


def _setup(model, size):
    import randomtilings_b200 as rt
    from randomtilings_b200.project import extremal_heights

    code = rt.RT_DOMINO if model == "domino" else rt.RT_LOZENGE
    d = rt.DominoTiler.AztecDiamond(size) if model == "domino" else rt.LozengeTiler.Hexagon(size, size + 3, size // 2)
    hmin, hmax = extremal_heights(code, d)
    return code, d, hmin, hmax


@pytest.mark.parametrize("model,size", [("domino", 13), ("domino", 100), ("domino", 300), ("lozenge", 10),
                                        ("lozenge", 60)])
def test_gpu_projection_matches_oracle(model, size):
    from randomtilings_b200.project import project_heights

    code, d, hmin, hmax = _setup(model, size)
    rng = np.random.default_rng(size)
    inside = hmin != INF
    n = int(round(hmin.size ** 0.5))
    ii, jj = np.divmod(np.arange(n * n), n)
    lo, hi = hmin.astype(np.float64), hmax.astype(np.float64)
    targets = [
        np.where(inside, (lo + hi) / 2 + 4 * np.sin(ii / 7.0) * np.cos(jj / 5.0), 0),
        np.where(inside, lo + (hi - lo) * rng.uniform(0, 1, n * n), 0),
        np.where(inside, (lo + hi) / 2 + rng.normal(0, 20, n * n), 0),
    ]
    for t in targets:
        t = t.astype(np.float32)
        got, st = project_heights(code, d, hmin, hmax, t)
        want = po.project_heights(model, d, hmin, hmax, t)
        assert np.array_equal(got, want), st
        if size <= 60:
            check_height_function(model, d, got, hmin, hmax)


def test_gpu_warm_tiling_is_a_tiling_of_the_domain():
    import randomtilings_b200 as rt
    from randomtilings_b200.project import warm_tiling

    code, d, hmin, hmax = _setup("domino", 40)
    t = warm_tiling(code, d, np.where(hmin != INF, (hmin.astype(np.float64) + hmax) / 2, 0).astype(np.float32))
    assert np.array_equal(rt.DominoTiler.TilingToDomain(t), d)
