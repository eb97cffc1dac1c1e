"""Host logic of the learned warm start (randomtilings_b200/warmstart.py):
domain specs, features, the fraction <-> height maps, training specs."""
from __future__ import annotations

import math

import numpy as np

from randomtilings_b200 import warmstart as ws


def test_training_specs_follow_the_ranges():
    specs = ws.training_specs(400, seed=3, aztec=(64, 1024), hexagon=(64, 512), q=(0.98, 1.0))
    az = [s for s in specs if s.kind == ws.AZTEC]
    hx = [s for s in specs if s.kind == ws.HEXAGON]
    assert len(az) == len(hx) == 200
    assert all(64 <= s.size[0] <= 1024 and s.q == 1.0 for s in az)
    assert all(64 <= v <= 512 for s in hx for v in s.size)
    assert all(0.98 <= s.q <= 1.0 for s in hx)
    assert ws.training_specs(400, seed=3) == ws.training_specs(400, seed=3)


def test_features_and_fraction_round_trip():
    for spec in (ws.DomainSpec(ws.AZTEC, (12,)), ws.DomainSpec(ws.HEXAGON, (5, 9, 7), 0.99)):
        p = ws.prepare(spec)
        x = ws.features(p)
        assert x.shape == (p.idx.size, 8) and x.dtype == np.float32
        assert x[:, 0].min() == -1 and x[:, 0].max() == 1 and x[:, 1].min() == -1 and x[:, 1].max() == 1
        assert np.all(x[:, 2] == (1 if spec.kind == ws.AZTEC else -1))
        if spec.kind == ws.AZTEC:
            assert np.all(x[:, 3] == 1) and np.all(x[:, 4:6] == 0)  # order 12: even
        else:
            assert np.allclose(x[0, 3:6], [3 * 5 / 21 - 1, 3 * 9 / 21 - 1, 3 * 7 / 21 - 1])
        assert np.allclose(x[:, 7], 16 / spec.side)
        if spec.q < 1:
            assert np.allclose(x[:, 6], -spec.side * math.log(spec.q))
        # heights between the extremal ones map to fractions and back
        assert np.all(p.hmin[p.idx] <= p.hmax[p.idx])
        mid = (p.hmin.astype(np.float64) + p.hmax) / 2
        f, live = ws.fraction(p, mid)
        assert np.allclose(f[live], 0.5)
        t = ws.heights_from_fraction(p, f)
        assert np.allclose(t[p.idx], mid[p.idx], atol=1e-3)
        f0, _ = ws.fraction(p, p.hmin.astype(np.float64))
        f1, _ = ws.fraction(p, p.hmax.astype(np.float64))
        assert np.all(f0[live] == 0) and np.all(f1[live] == 1)


def test_burn_in_scales_with_the_side_squared():
    a = ws.burn_sweeps(ws.DomainSpec(ws.AZTEC, (100,)))
    b = ws.burn_sweeps(ws.DomainSpec(ws.AZTEC, (200,)))
    assert b == 4 * a
    assert ws.burn_sweeps(ws.DomainSpec(ws.HEXAGON, (30, 30, 30))) == int(7.0 * 900)
