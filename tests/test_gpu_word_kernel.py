"""The word-parallel kernel of the int8 models (rt_word.cu) and the generic
walk kernel (rt_walk.cu) both produce the oracle's bytes.  RT_WALK_KERNEL
selects the kernel and RT_WALK_CTAS the word kernel's grid when a handle is
created; the cases cover one to four words per thread and bands of one row."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["generic", "word"])
def kernel(request, monkeypatch):
    monkeypatch.setenv("RT_WALK_KERNEL", request.param)
    return request.param


def _walk(tiler, t, steps, seed):
    a = np.array(t, dtype=np.int32)
    tiler.Walk(a, steps, seed)
    return a


@pytest.mark.parametrize("order", [3, 13, 100])
@pytest.mark.parametrize("cftp", [False, True])
def test_domino(kernel, order, cftp):
    import randomtilings_b200 as rt

    t = golden("builders")[f"domino/aztec{order}/min"]
    got = _walk(rt.DominoTiler(kernel=int(cftp)), t, 1500, 42)
    assert np.array_equal(got, po.domino_walk(t, 1500, 42, cftp=cftp))


@pytest.mark.parametrize("key", ["hex2_0", "hex4_1", "hex13_5", "hex20_0"])
def test_lozenge(kernel, key):
    import randomtilings_b200 as rt

    t = golden("builders")[f"lozenge/{key}/max"]
    got = _walk(rt.LozengeTiler(), t, 1500, 5)
    assert np.array_equal(got, po.lozenge_walk(t, 1500, 5))


@pytest.mark.parametrize("model", ["domino", "domino_cftp", "lozenge"])
def test_fast_mode(kernel, model):
    import randomtilings_b200 as rt

    b = golden("builders")
    if model.startswith("domino"):
        t = b["domino/aztec100/max"]
        tl = rt.DominoTiler(kernel=int(model == "domino_cftp"), rng=rt.RT_RNG_PHILOX)
    else:
        t = b["lozenge/hex20_0/min"]
        tl = rt.LozengeTiler(rng=rt.RT_RNG_PHILOX)
    got = _walk(tl, t, 1200, 2**33 + 17)
    assert np.array_equal(got, po.walk_fast(model, t, 1200, 2**33 + 17))


@pytest.mark.parametrize("ctas", [1, 3, 4, 7, 31, 204])
def test_word_kernel_grids(monkeypatch, ctas):
    """Bands of a whole lattice down to one row per CTA; Aztec 100 (204 rows of
    26 words) puts 4 words on every thread at 3 and 4 CTAs, 2 at 7, 1 at 31."""
    import randomtilings_b200 as rt

    monkeypatch.setenv("RT_WALK_KERNEL", "word")
    monkeypatch.setenv("RT_WALK_CTAS", str(ctas))
    t = golden("builders")["lozenge/hex20_0/max"]
    got = _walk(rt.LozengeTiler(), t, 900, 3)
    assert np.array_equal(got, po.lozenge_walk(t, 900, 3))
    t = golden("builders")["domino/aztec100/min" if ctas >= 3 else "domino/aztec13/min"]
    got = _walk(rt.DominoTiler(), t, 900, 3)
    assert np.array_equal(got, po.domino_walk(t, 900, 3))


@pytest.mark.parametrize("ctas", [1, 2, 3, 7])
def test_word_kernel_grids_fast_mode(monkeypatch, ctas):
    """Fast mode on Aztec 100: 5304 words on one CTA (walked at run time),
    2652 (4 per thread), 1768 (2 per thread), 780 (1 per thread)."""
    import randomtilings_b200 as rt

    monkeypatch.setenv("RT_WALK_KERNEL", "word")
    monkeypatch.setenv("RT_WALK_CTAS", str(ctas))
    t = golden("builders")["domino/aztec100/max"]
    for kernel, model in ((0, "domino"), (1, "domino_cftp")):
        got = _walk(rt.DominoTiler(kernel=kernel, rng=rt.RT_RNG_PHILOX), t, 700, 8)
        assert np.array_equal(got, po.walk_fast(model, t, 700, 8))


def test_word_kernel_cftp(monkeypatch):
    import randomtilings_b200 as rt

    monkeypatch.setenv("RT_WALK_KERNEL", "word")
    b = golden("builders")
    tmax, tmin = b["domino/aztec13/max"], b["domino/aztec13/min"]
    got, st = rt.DominoTiler(kernel=1).CFTP(tmax, tmin, first_steps=64, master_seed=99, max_trials=20)
    want, trials, total, ok = po.cftp(tmax, tmin, 64, 99, max_trials=20)
    assert st["coalesced"] and ok and st["total_steps"] == total
    assert np.array_equal(got, want)
