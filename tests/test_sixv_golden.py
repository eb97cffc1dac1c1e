"""The six-vertex restatement reproduces its committed regression vectors
(tests/golden/sixv.npz, written by tests/golden/make_sixv_golden.py): walks
from both domain-wall extremes, uniform and weighted, epoch walks and CFTP
samples with their trial counts.  No GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po

WEIGHTED = (1.0, 0.7, 1.6, 1.2, 2.0, 0.5)


@pytest.mark.parametrize("n", [7, 24, 65])
def test_walks_and_epochs(n):
    z = golden("sixv")
    lo, hi = po.sixv_dwbc(n)
    for sname, start in (("min", lo), ("max", hi)):
        for wname, w in (("uniform", po.SIXV_UNIFORM), ("weighted", WEIGHTED)):
            got = po.sixv_walk(start, 40, 0x5EED + n, chain=n % 3, w=w)
            assert np.array_equal(got, z[f"walk/{n}/{sname}/{wname}"]), (sname, wname)
    assert np.array_equal(po.sixv_walk(lo, [5, 11, 2], [3, 2**40 + 9, 77]), z[f"epochs/{n}"])


@pytest.mark.parametrize("n,seed", [(6, 0), (10, 4), (16, 1)])
def test_cftp(n, seed):
    z = golden("sixv")
    h, trials, sweeps, ok = po.sixv_cftp(n, 4, seed)
    assert ok
    assert np.array_equal(h, z[f"cftp/{n}/{seed}"])
    assert [trials, sweeps] == z[f"cftp/{n}/{seed}/counts"].tolist()
