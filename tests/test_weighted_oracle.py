"""The oracle's weighted domino heat bath (orc_domino_walk_weighted, the
checker of rt_set_domino_weights): equal weights give the reference's
unweighted heat bath bit for bit (TinyMT single and epoch walks, Philox),
and with unequal weights the chain's stationary law is the weighted one,
P(T) proportional to the product of T's domino weights, checked on the
Aztec diamond of order 2 (8 tilings).  CPU only."""
from __future__ import annotations

from collections import Counter

import numpy as np
import pytest
from scipy import stats

from conftest import golden
from oracle import pyoracle as po

WH = np.array([[1.0, 0.3], [0.5, 2.0]])
WV = np.array([[0.7, 1.5], [1.0, 0.2]])


def tiling_weight(t, wh, wv):
    """Product of the domino weights: a horizontal domino once, at the vertex
    whose up edge it crosses (bit 1: top-left square (i-1, j-1)); a vertical
    one at the vertex whose edge towards j+1 it crosses (bit 8: (i-1, j))."""
    t = np.asarray(t).reshape(-1)
    n = int(round(t.size ** 0.5))
    p = wh.shape[0]
    w = 1.0
    for i in range(n):
        for j in range(n):
            v = int(t[i * n + j])
            if v & 1:
                w *= wh[(i - 1) % p, (j - 1) % p]
            if v & 8:
                w *= wv[(i - 1) % p, j % p]
    return w


@pytest.mark.parametrize("period", [1, 2, 4])
def test_equal_weights_are_the_reference_heat_bath(period):
    t = golden("builders")["domino/aztec13/min"]
    one = np.full((period, period), 1.3)
    assert np.array_equal(po.domino_walk_weighted(t, [700], [5], one, one, single_walk=True),
                          po.domino_walk(t, 700, 5, cftp=True))
    assert np.array_equal(po.domino_walk_weighted(t, [300, 200], [5, 9], one, one),
                          po.domino_walk_epochs(t, [300, 200], [5, 9], cftp=True))
    assert np.array_equal(po.domino_walk_weighted(t, [300, 200], [5, 2**40 + 1], one, one, fast=True),
                          po.walk_fast("domino_cftp", t, [300, 200], [5, 2**40 + 1]))


def test_unequal_weights_change_the_walk():
    t = golden("builders")["domino/aztec13/min"]
    assert not np.array_equal(po.domino_walk_weighted(t, [700], [5], WH, WV, single_walk=True),
                              po.domino_walk(t, 700, 5, cftp=True))


def test_stationary_law_is_the_weighted_one():
    t0 = golden("builders")["domino/aztec2/min"]
    ends = [po.domino_walk_weighted(t0, [200], [key], WH, WV, fast=True) for key in range(4000)]
    c = Counter(e.tobytes() for e in ends)
    assert len(c) == 8
    keys = sorted(c)
    w = np.array([tiling_weight(np.frombuffer(k, dtype=np.int32), WH, WV) for k in keys])
    obs = np.array([c[k] for k in keys], dtype=float)
    assert stats.chisquare(obs, obs.sum() * w / w.sum()).pvalue > 1e-4
    assert stats.chisquare(obs).pvalue < 1e-6  # not the uniform law


def _p12(wh, wv, i, j):
    p = wh.shape[0]
    w3 = wh[(i - 1) % p, (j - 1) % p] * wh[i % p, (j - 1) % p]
    w12 = wv[(i - 1) % p, (j - 1) % p] * wv[(i - 1) % p, j % p]
    return w12 / (w3 + w12)


def test_two_periodic_weights():
    import randomtilings_b200 as rt

    a, b = 1.0, 0.5
    wh, wv = rt.DominoTiler.TwoPeriodicWeights(a, b)
    odd = set()
    for i in range(4):
        for j in range(4):
            if (i + j) % 2 == 0:
                assert _p12(wh, wv, i, j) == 0.5  # even faces: all four dominoes share one weight
            else:
                odd.add(round(_p12(wh, wv, i, j), 12))
    assert odd == {round(a * a / (a * a + b * b), 12), round(b * b / (a * a + b * b), 12)}
    u, v = rt.DominoTiler.TwoPeriodicWeights(0.7, 0.7)
    assert np.all(u == 0.7) and np.all(v == 0.7)


# ---- lozenges ----
LW = (np.array([[1.0, 0.4], [1.6, 0.8]]), np.array([[0.5, 1.2], [2.0, 1.0]]), np.array([[1.5, 0.7], [0.9, 1.1]]))


def lozenge_tiling_weight(t, w0, w1, w2):
    """Product of the lozenge weights: each lozenge once, at the lower end
    (i, j) of the edge it covers: bit 8 (edge to (i, j+1)) -> w0, bit 2 (to
    (i-1, j+1)) -> w1, bit 1 (to (i-1, j)) -> w2."""
    t = np.asarray(t).reshape(-1)
    n = int(round(t.size ** 0.5))
    p = w0.shape[0]
    w = 1.0
    for i in range(n):
        for j in range(n):
            v = int(t[i * n + j])
            for bit, table in ((8, w0), (2, w1), (1, w2)):
                if v & bit:
                    w *= table[i % p, j % p]
    return w


@pytest.mark.parametrize("period", [1, 2, 4])
def test_equal_lozenge_weights_are_the_reference_rule(period):
    t = golden("builders")["lozenge/hex10_2/max"]
    one = np.full((period, period), 0.9)
    assert np.array_equal(po.lozenge_walk_weighted(t, [300, 200], [5, 9], one, one, one),
                          po.lozenge_walk_epochs(t, [300, 200], [5, 9]))
    assert np.array_equal(po.lozenge_walk_weighted(t, [500], [5 + 2**40], one, one, one, fast=True),
                          po.walk_fast("lozenge", t, [500], [5 + 2**40]))


def test_lozenge_stationary_law_is_the_weighted_one():
    import randomtilings_b200 as rt

    t0 = np.asarray(rt.LozengeTiler.MinTiling(rt.LozengeTiler.Hexagon(2, 2, 2)))
    ends = [po.lozenge_walk_weighted(t0, [300], [key], *LW, fast=True) for key in range(4000)]
    c = Counter(e.tobytes() for e in ends)
    assert len(c) == 20  # plane partitions in a 2 x 2 x 2 box
    keys = sorted(c)
    w = np.array([lozenge_tiling_weight(np.frombuffer(k, dtype=np.int32), *LW) for k in keys])
    obs = np.array([c[k] for k in keys], dtype=float)
    assert stats.chisquare(obs, obs.sum() * w / w.sum()).pvalue > 1e-4
    assert stats.chisquare(obs).pvalue < 1e-6
