"""Batched chains (include/rt_b200_batch.h) on the GPU: every chain equals
its single-chain fast-mode walk (and the oracle's replay), whatever the
cluster size the plan uses; runs compose; the autotuner does not advance the
chains."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

SWEEPS = 7


def _chains(rt):
    b = golden("builders")
    D, L, R, T = rt.RT_DOMINO, rt.RT_LOZENGE, rt.RT_RECTTRI, rt.RT_TRIDIMER
    return [
        (D, 0, b["domino/aztec13/min"], 11, "domino"),
        (D, 1, b["domino/aztec13/max"], 12, "domino_cftp"),
        (D, 0, rt.DominoTiler.MinTiling(rt.DominoTiler.AztecDiamond(40)), 2**40 + 5, "domino"),
        (L, 0, rt.LozengeTiler.MinTiling(rt.LozengeTiler.Hexagon(5, 7, 9)), 13, "lozenge"),
        (L, 0, rt.LozengeTiler.MaxTiling(rt.LozengeTiler.Hexagon(20, 3, 11)), 14, "lozenge"),
        (L, 0, b["lozenge/hex20_0/min"], 15, "lozenge"),
        (R, 0, b["recttri/min_hex9"], 16, "recttri"),
        (R, 0, b["recttri/max_hex20"], 17, "recttri"),
        (T, 0, rt.TriangleDimerTiler.IceCreamCone(12, 0), 18, "tridimer"),
        (T, 0, rt.TriangleDimerTiler.IceCreamCone(25, 7), 19, "tridimer"),
        (T, 0, rt.TriangleDimerTiler.BiboneHexagon(7), 20, "tridimer"),
    ]


def _tiler(rt, model, kernel, chain):
    cls = {rt.RT_DOMINO: rt.DominoTiler, rt.RT_LOZENGE: rt.LozengeTiler, rt.RT_RECTTRI: rt.RectTriangleTiler,
           rt.RT_TRIDIMER: rt.TriangleDimerTiler}[model]
    return cls(kernel=kernel, rng=rt.RT_RNG_PHILOX, chain=chain)


def _run_batch(rt, chains, sweeps=SWEEPS, tuning=None, split=None):
    bt = rt.Batch()
    for c, (model, kernel, t, key, _) in enumerate(chains):
        assert bt.add(model, t, key, chain=c, kernel=kernel) == c
    if tuning is not None:
        bt.set_tuning(*tuning)
    for s in (split or [sweeps]):
        bt.run(s)
    out = [bt.download(c) for c in range(len(chains))]
    info = bt.info()
    bt.close()
    return out, info


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


@pytest.fixture(scope="module")
def singles(rt):
    from randomtilings_b200.batch import STEPS_PER_SWEEP

    out = []
    for c, (model, kernel, t, key, _) in enumerate(_chains(rt)):
        a = np.array(t, dtype=np.int32)
        _tiler(rt, model, kernel, c).Walk(a, SWEEPS * STEPS_PER_SWEEP[model], key)
        out.append(a)
    return out


def test_single_fast_walks_with_a_chain_index_match_the_oracle(rt, singles):
    from randomtilings_b200.batch import STEPS_PER_SWEEP

    for c, (model, kernel, t, key, name) in enumerate(_chains(rt)):
        want = po.walk_fast(name, t, SWEEPS * STEPS_PER_SWEEP[model], key, chain=c)
        assert np.array_equal(singles[c], want), name


@pytest.mark.parametrize("cluster", [1, 2, 4])
@pytest.mark.parametrize("block", [128, 1024])
def test_batch_equals_single_chain_walks(rt, singles, cluster, block):
    out, info = _run_batch(rt, _chains(rt), tuning=(False, cluster, block))
    for c, got in enumerate(out):
        assert np.array_equal(got, singles[c]), (c, info)
    assert all(p["cluster"] == cluster for p in info["plans"].values())


def test_autotuned_batch_equals_single_chain_walks(rt, singles):
    out, info = _run_batch(rt, _chains(rt))
    for c, got in enumerate(out):
        assert np.array_equal(got, singles[c]), (c, info)
    assert info["tune_ms"] > 0 and set(info["plans"]) == {"domino", "domino_heat_bath", "lozenge", "rect_triangle",
                                                           "triangle_dimer"}


def test_batch_runs_compose(rt, singles):
    out, _ = _run_batch(rt, _chains(rt), tuning=(False, 2, 256), split=[3, 4])
    for c, got in enumerate(out):
        assert np.array_equal(got, singles[c])


@pytest.mark.parametrize("spl", [3, 4])
def test_sweeps_per_launch_compose(rt, singles, spl):
    """A run split into launches of `spl` sweeps (plus one shorter launch for
    the rest) equals the single-chain walks."""
    bt = rt.Batch()
    for model, kernel, t, key, _ in _chains(rt):
        bt.add(model, t, key=key, chain=len(bt), kernel=kernel)
    bt.set_sweeps_per_launch(spl)
    bt.run(SWEEPS)
    assert all(p["sweeps_per_launch"] == spl for p in bt.info()["plans"].values())
    for c in range(len(bt)):
        assert np.array_equal(bt.download(c), singles[c]), c
    bt.close()


def test_mixed_workload_chains(rt):
    """The first chains of the mixed benchmark workload (Aztec diamonds up to
    order 256 need 2-CTA clusters), two sweeps."""
    from randomtilings_b200 import workloads
    from randomtilings_b200.batch import STEPS_PER_SWEEP

    chains = []
    for seed in range(8):
        model, t = workloads.mixed_chain(seed)
        chains.append((model, 0, t, seed, None))
    out, info = _run_batch(rt, chains, sweeps=2)
    for c, (model, kernel, t, key, _) in enumerate(chains):
        a = np.array(t, dtype=np.int32)
        _tiler(rt, model, kernel, c).Walk(a, 2 * STEPS_PER_SWEEP[model], key)
        assert np.array_equal(out[c], a), (c, info)
    assert info["plans"]["domino"]["cluster"] >= 2


def test_batch_rejects_unsupported_chains(rt):
    bt = rt.Batch()
    with pytest.raises(rt.RtError):
        bt.add(rt.RT_LOZENGE, golden("builders")["lozenge/hex4_0/min"], 1, kernel=rt.RT_KERNEL_QWEIGHT)
    with pytest.raises(rt.RtError):
        bt.add(rt.RT_DOMINO, np.zeros(49, dtype=np.int32), 1)


def test_volume_weighted_lozenge_chains_equal_the_oracle(rt):
    """Per-chain volume weight q (rt_chain.q) on the int8 lozenge family:
    each chain equals the oracle's replay of the same rule and draws, and q = 1
    equals the uniform chain."""
    tmin = rt.LozengeTiler.MinTiling(rt.LozengeTiler.Hexagon(11, 8, 14))
    qs = [np.float32(0.985), np.float32(0.5), np.float32(1.0), np.float32(0.0)]
    bt = rt.Batch()
    for c, qv in enumerate(qs):
        bt.add(rt.RT_LOZENGE, tmin, key=77, chain=c, q=float(qv))
    bt.run(SWEEPS)
    got = [bt.download(c) for c in range(len(qs))]
    bt.close()
    for c, qv in enumerate(qs):
        q = 1.0 if qv == 0 else float(qv)
        want = po.walk_fast("lozenge_q8", tmin, 3 * SWEEPS, 77, chain=c, q=q)
        assert np.array_equal(got[c], want), c
    assert np.array_equal(po.walk_fast("lozenge_q8", tmin, 3 * SWEEPS, 77, chain=3, q=1.0),
                          po.walk_fast("lozenge", tmin, 3 * SWEEPS, 77, chain=3))
    # q = 0.5 removes cubes twice as often as it adds them: the volume ends lower
    assert not np.array_equal(got[1], got[2])


def test_batch_rejects_bad_q(rt):
    bt = rt.Batch()
    t = rt.LozengeTiler.MinTiling(rt.LozengeTiler.Hexagon(4, 4, 4))
    with pytest.raises(rt.RtError):
        bt.add(rt.RT_LOZENGE, t, key=1, q=1.5)
    with pytest.raises(rt.RtError):
        bt.add(rt.RT_DOMINO, rt.DominoTiler.MinTiling(rt.DominoTiler.AztecDiamond(5)), key=1, q=0.9)
    bt.close()
