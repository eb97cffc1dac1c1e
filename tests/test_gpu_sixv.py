"""The six-vertex model on the GPU (include/rt_b200_sixv.h) against its
restatement (oracle/sixv_oracle.c): walks bit-equal for several sizes, keys,
chains and weights; CFTP equal to the oracle's composition and its exact
samples uniform over the alternating-sign matrices."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

WEIGHTED = (1.0, 0.7, 1.6, 1.2, 2.0, 0.5)


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


@pytest.mark.parametrize("n,sweeps,key,chain", [(2, 5, 1, 0), (4, 40, 7, 0), (9, 100, 2**40 + 3, 5),
                                                (37, 300, 11, 1), (200, 150, 42, 0), (515, 20, 99, 3)])
@pytest.mark.parametrize("w", [po.SIXV_UNIFORM, WEIGHTED])
def test_walk_matches_restatement(rt, n, sweeps, key, chain, w):
    tl = rt.SixVertexTiler(weights=w)
    for start in (rt.SixVertexTiler.MinHeights(n), rt.SixVertexTiler.MaxHeights(n)):
        h = start.copy()
        tl.Walk(h, sweeps, key, chain)
        assert rt.SixVertexTiler.IsValid(h)
        assert np.array_equal(h, po.sixv_walk(start, sweeps, key, chain=chain, w=w))
    tl.close()


def test_thresholds_match_restatement(rt):
    tl = rt.SixVertexTiler(weights=WEIGHTED)
    thr, mono = tl.Thresholds()
    assert np.array_equal(thr, po.sixv_thresholds(WEIGHTED))
    tl.close()


@pytest.mark.parametrize("n,seed", [(5, 0), (12, 3), (40, 1)])
def test_cftp_matches_restatement(rt, n, seed):
    tl = rt.SixVertexTiler()
    h, st = tl.CFTP(n, first_sweeps=8, master_seed=seed)
    want, trials, sweeps, ok = po.sixv_cftp(n, 8, seed)
    assert st["coalesced"] and ok
    assert st["trials"] == trials and st["sweeps"] == sweeps
    assert np.array_equal(h, want)
    tl.close()


def test_cftp_samples_are_uniform(rt):
    n, runs = 3, 1400
    confs = po.sixv_enumerate(n)
    index = {c.tobytes(): k for k, c in enumerate(confs)}
    cnt = np.zeros(len(confs))
    tl = rt.SixVertexTiler()
    for s in range(runs):
        h, st = tl.CFTP(n, first_sweeps=2, master_seed=s)
        cnt[index[h.tobytes()]] += 1
    tl.close()
    e = runs / len(confs)
    assert float(((cnt - e) ** 2 / e).sum()) < 25.0


def test_large_walk_stays_valid(rt):
    n = 1000
    tl = rt.SixVertexTiler()
    h = rt.SixVertexTiler.MinHeights(n)
    tl.Walk(h, 200, 5)
    assert rt.SixVertexTiler.IsValid(h)
    a = rt.SixVertexTiler.HeightsToASM(h)
    assert (a.sum(axis=0) == 1).all() and (a.sum(axis=1) == 1).all()
    tl.close()


def test_wide_walk_matches_restatement(rt):
    """n = 6000: the bands do not fit shared memory, so the walk takes one
    launch per colour step; the result is the restatement's all the same."""
    n = 6000
    start = rt.SixVertexTiler.MinHeights(n)
    h = start.copy()
    tl = rt.SixVertexTiler()
    tl.Walk(h, 1, 77, 2)
    tl.close()
    assert np.array_equal(h, po.sixv_walk(start, 1, 77, chain=2))


def test_bench_walk_matches_restatement(rt):
    """The walk the benchmark times (n = 1000, 400 sweeps from the minimal
    heights, key 2): many bands, every halo exchange of a long launch."""
    n = 1000
    start = rt.SixVertexTiler.MinHeights(n)
    h = start.copy()
    tl = rt.SixVertexTiler()
    tl.Walk(h, 400, 2)
    tl.close()
    assert np.array_equal(h, po.sixv_walk(start, 400, 2))


@pytest.mark.parametrize("n", [7, 24, 65])
def test_walks_match_the_committed_vectors(rt, n):
    """The CUDA walk against tests/golden/sixv.npz directly (the vectors the
    restatement is held to), from both extremes, uniform and weighted."""
    from conftest import golden

    z = golden("sixv")
    for w, wname in ((po.SIXV_UNIFORM, "uniform"), (WEIGHTED, "weighted")):
        tl = rt.SixVertexTiler(weights=w)
        for sname, start in (("min", rt.SixVertexTiler.MinHeights(n)), ("max", rt.SixVertexTiler.MaxHeights(n))):
            h = start.copy()
            tl.Walk(h, 40, 0x5EED + n, n % 3)
            assert np.array_equal(h, z[f"walk/{n}/{sname}/{wname}"]), (sname, wname)
        tl.close()
