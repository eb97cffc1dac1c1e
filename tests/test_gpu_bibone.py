"""Triangle-dimer walks on the bibone hexagon (rt_tridimer_hexagon) on the
GPU: the bit-exact walk equals the oracle's (which the reference's own walk
equals on this domain, tests/test_bibone_hexagon.py), and the fast mode
equals the oracle's replay, at the batched workload's side 64 too."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


@pytest.mark.parametrize("s,steps,seed", [(6, 2000, 3), (20, 1000, 42), (64, 300, 7)])
def test_bit_exact_walk(rt, s, steps, seed):
    t = np.asarray(rt.TriangleDimerTiler.BiboneHexagon(s), dtype=np.int32)
    a = t.copy()
    rt.TriangleDimerTiler().Walk(a, steps, seed)
    assert np.array_equal(a, po.tridimer_walk(t, steps, seed))


@pytest.mark.parametrize("s,steps,key", [(9, 900, 5), (64, 300, 11)])
def test_fast_walk(rt, s, steps, key):
    t = np.asarray(rt.TriangleDimerTiler.BiboneHexagon(s), dtype=np.int32)
    a = t.copy()
    rt.TriangleDimerTiler(rng=rt.RT_RNG_PHILOX).Walk(a, steps, key)
    assert np.array_equal(a, po.walk_fast("tridimer", t, steps, key))
