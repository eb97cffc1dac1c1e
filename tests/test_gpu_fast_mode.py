"""Fast mode (RT_RNG_PHILOX) on the GPU, through the C ABI: bit-equal with
the oracle's replay of the same counter-based draws and colour cycle, CFTP in
fast mode against the oracle's, and the stationary law against exact
enumeration and against the bit-exact mode's samples."""
from __future__ import annotations

from collections import Counter

import numpy as np
import pytest
from scipy import stats

from conftest import golden
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


def _fast(rt, cls, **kw):
    from randomtilings_b200 import _capi

    return cls(rng=_capi.RT_RNG_PHILOX, **kw)


def _walk(tiler, t, steps, seed):
    a = np.array(t, dtype=np.int32)
    tiler.Walk(a, steps, seed)
    return a


@pytest.mark.parametrize("order", [3, 13, 100])
@pytest.mark.parametrize("kernel", [0, 1])
def test_domino_fast_matches_oracle(rt, order, kernel):
    t = golden("builders")[f"domino/aztec{order}/min"]
    got = _walk(_fast(rt, rt.DominoTiler, kernel=kernel), t, 1001, 42 + (7 << 32))
    want = po.walk_fast("domino_cftp" if kernel else "domino", t, 1001, 42 + (7 << 32))
    assert np.array_equal(got, want)


def test_domino_fast_epochs_match_oracle(rt):
    t = golden("builders")["domino/aztec13/max"]
    tl = _fast(rt, rt.DominoTiler, kernel=1)
    a = np.array(t, dtype=np.int32)
    tl.Walk(a, [300, 200, 57], [11, 2**40 + 3, 5])
    assert np.array_equal(a, po.walk_fast("domino_cftp", t, [300, 200, 57], [11, 2**40 + 3, 5]))


@pytest.mark.parametrize("key", ["hex4_1", "hex13_5", "hex20_0"])
def test_lozenge_fast_matches_oracle(rt, key):
    t = golden("builders")[f"lozenge/{key}/min"]
    got = _walk(_fast(rt, rt.LozengeTiler), t, 2000, 9)
    assert np.array_equal(got, po.walk_fast("lozenge", t, 2000, 9))


@pytest.mark.parametrize("qcmp", [0, 1])
@pytest.mark.parametrize("q", [0.99, 0.5, 1.3])
def test_qlozenge_fast_matches_oracle(rt, q, qcmp):
    t = golden("builders")["lozenge/hex13_5/max"]
    got = _walk(_fast(rt, rt.LozengeTiler, kernel=2, q=q, qcmp=qcmp), t, 1500, 3)
    assert np.array_equal(got, po.walk_fast("qlozenge", t, 1500, 3, q=q, qcmp_double=bool(qcmp)))


def test_recttri_fast_matches_oracle(rt):
    w = np.array([0.0, 1.0, 2.0, 0.5, 1.5, 0.7, 1.1, 1.5, 0.7, 1.1, 0.3, 3.0, 1.0, 0.3, 3.0, 1.0], dtype=np.float32)
    b = golden("builders")
    for key, weights in (("recttri/min_hex9", None), ("recttri/slope_hex9", w), ("recttri/max_hex20", None)):
        t = b[key]
        kw = {} if weights is None else {"weights": weights}
        got = _walk(_fast(rt, rt.RectTriangleTiler, **kw), t, 1200, 77)
        assert np.array_equal(got, po.walk_fast("recttri", t, 1200, 77, weights=weights)), key


@pytest.mark.parametrize("n,m", [(12, 0), (25, 7), (40, 10)])
def test_tridimer_fast_matches_oracle(rt, n, m):
    t = rt.TriangleDimerTiler.IceCreamCone(n, m)
    got = _walk(_fast(rt, rt.TriangleDimerTiler), t, 900, 1234)
    assert np.array_equal(got, po.walk_fast("tridimer", t, 900, 1234))


@pytest.mark.parametrize("model,order_or_hex,first", [("domino_cftp", 13, 64), ("lozenge", "hex10_2", 64),
                                                      ("qlozenge", "hex10_2", 64)])
def test_fast_cftp_matches_oracle(rt, model, order_or_hex, first):
    b = golden("builders")
    if model == "domino_cftp":
        tmax, tmin = b[f"domino/aztec{order_or_hex}/max"], b[f"domino/aztec{order_or_hex}/min"]
        tl = _fast(rt, rt.DominoTiler, kernel=1)
    else:
        tmax, tmin = b[f"lozenge/{order_or_hex}/max"], b[f"lozenge/{order_or_hex}/min"]
        tl = _fast(rt, rt.LozengeTiler, kernel=2 if model == "qlozenge" else 0, q=0.9)
    kw = {"q": 0.9} if model == "qlozenge" else {}
    got, st = tl.CFTP(tmax, tmin, first_steps=first, master_seed=2024, max_trials=20)
    want, trials, total, ok = po.cftp(tmax, tmin, first, 2024, model=model, fast=True, max_trials=20, **kw)
    assert st["coalesced"] and ok and st["trials"] == trials and st["total_steps"] == total
    assert np.array_equal(got, want)


def test_bit_exact_lozenge_cftp_matches_oracle(rt):
    b = golden("builders")
    tmax, tmin = b["lozenge/hex10_2/max"], b["lozenge/hex10_2/min"]
    got, st = rt.LozengeTiler().CFTP(tmax, tmin, first_steps=64, master_seed=5, max_trials=20)
    want, trials, total, ok = po.cftp(tmax, tmin, 64, 5, model="lozenge", max_trials=20)
    assert st["coalesced"] and ok and st["total_steps"] == total
    assert np.array_equal(got, want)


def _counts(samples):
    return Counter(s.tobytes() for s in samples)


# The statistical tests are deterministic (fixed keys and seeds); a law that
# is right fails them with probability 1e-4 (the p-value threshold).
P_MIN = 1e-4


def test_fast_chains_and_cftp_are_uniform_on_aztec3(rt):
    """Aztec diamond of order 3: 2^6 = 64 domino tilings.  Fast-mode chain
    ends (independent keys) and fast-mode CFTP samples are both uniform."""
    b = golden("builders")
    tmax, tmin = b["domino/aztec3/max"], b["domino/aztec3/min"]
    tl = _fast(rt, rt.DominoTiler, kernel=1)
    ends = [_walk(tl, tmin, 200, key) for key in range(6400)]
    c = _counts(ends)
    assert len(c) == 64 and stats.chisquare(list(c.values())).pvalue > P_MIN
    samples = [tl.CFTP(tmax, tmin, first_steps=16, master_seed=s)[0] for s in range(6400)]
    c = _counts(samples)
    assert len(c) == 64 and stats.chisquare(list(c.values())).pvalue > P_MIN


def test_fast_q_lozenge_law_equals_bit_exact_mode(rt):
    """q = 0.7 on the 2 x 2 x 2 hexagon (20 tilings): fast-mode chain ends
    and bit-exact-mode CFTP samples (the reference's update rule) have the
    same law (two-sample chi-square)."""
    b = golden("builders")
    tmax, tmin = b["lozenge/hex2_0/max"], b["lozenge/hex2_0/min"]
    fast = _fast(rt, rt.LozengeTiler, kernel=2, q=0.7)
    exact = rt.LozengeTiler(kernel=2, q=0.7)
    a = _counts(_walk(fast, tmin, 150, key) for key in range(4000))
    c = _counts(exact.CFTP(tmax, tmin, first_steps=32, master_seed=s)[0] for s in range(4000))
    keys = sorted(set(a) | set(c))
    assert len(keys) == 20
    table = np.array([[a.get(k, 0) for k in keys], [c.get(k, 0) for k in keys]])
    assert stats.chi2_contingency(table).pvalue > P_MIN
    # and q < 1 really tilts the law away from uniform
    assert stats.chisquare(table[0]).pvalue < 1e-6


def test_fast_mode_handles_lattices_too_large_for_bit_exact_mode(rt):
    """Aztec order 2000 (N = 4006, 8,012,004 positions) fits the fast mode's
    shared-memory-resident walk: it keeps no per-position generator state."""
    d = rt.DominoTiler.AztecDiamond(2000)
    t = rt.DominoTiler.MinTiling(d)
    got = _walk(_fast(rt, rt.DominoTiler), t, 20, 1)
    assert not np.array_equal(got, t)
    h = rt.DominoTiler.TilingToHeightfunc(got, d)
    assert np.array_equal(rt.DominoTiler.HeightfuncToTiling(h, d), got)
