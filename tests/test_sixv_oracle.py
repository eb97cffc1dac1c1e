"""The six-vertex restatement (oracle/sixv_oracle.c) against exact
enumeration, on the CPU.

The reference names the six-vertex model (README.md:3) without code, so its
oracle is this project's own statement of the model, pinned here: the
domain-wall height functions of the n x n grid are the alternating-sign
matrices (1, 2, 7, 42, 429 of them), the weight with c = sqrt 2 sums to the
2-enumeration 2^(n(n-1)/2) sqrt(2)^n, and the heat bath's samples follow the
exact law of the weights (chi-square over all 42 states of n = 4).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import pyoracle as po


@pytest.mark.parametrize("n,count", [(1, 1), (2, 2), (3, 7), (4, 42), (5, 429)])
def test_enumeration_counts_alternating_sign_matrices(n, count):
    confs = po.sixv_enumerate(n)
    assert len(confs) == count
    assert all((po.sixv_vertex_types(h) >= 0).all() for h in confs)


@pytest.mark.parametrize("n", [2, 3, 4, 5])
def test_two_enumeration(n):
    w = (1, 1, 1, 1, math.sqrt(2), math.sqrt(2))
    z = sum(po.sixv_weight(h, w) for h in po.sixv_enumerate(n))
    assert z == pytest.approx(2 ** (n * (n - 1) / 2) * math.sqrt(2) ** n)


def test_extremes_are_the_identity_and_anti_identity():
    lo, hi = po.sixv_dwbc(5)
    t_lo, t_hi = po.sixv_vertex_types(lo), po.sixv_vertex_types(hi)
    assert (t_lo >= 0).all() and (t_hi >= 0).all()
    # c-type vertices (4, 5) are the non-zero entries: the diagonals
    assert np.array_equal(np.argwhere(t_lo >= 4), np.argwhere(np.eye(5)))
    assert np.array_equal(np.argwhere(t_hi >= 4), np.argwhere(np.fliplr(np.eye(5))))


def test_uniform_thresholds_are_one_half():
    assert (po.sixv_thresholds() == 1 << 22).all()


@pytest.mark.parametrize("w", [(1, 1, 1, 1, 1, 1), (1.0, 0.7, 1.6, 1.2, 2.0, 0.5)])
def test_heat_bath_samples_the_weights(w):
    n, runs = 4, 6000
    confs = po.sixv_enumerate(n)
    index = {c.tobytes(): k for k, c in enumerate(confs)}
    p = np.array([po.sixv_weight(c, w) for c in confs])
    p /= p.sum()
    lo, _ = po.sixv_dwbc(n)
    cnt = np.zeros(len(confs))
    for r in range(runs):
        cnt[index[po.sixv_walk(lo, 60, r * 7919 + 13, w=w).tobytes()]] += 1
    chi2 = float(((cnt - runs * p) ** 2 / (runs * p)).sum())
    assert chi2 < 80.0, chi2  # 41 degrees of freedom: P(chi2 > 80) < 3e-4


def test_cftp_gives_valid_states_and_couples():
    for seed in range(5):
        h, trials, sweeps, ok = po.sixv_cftp(6, 8, seed)
        assert ok and (po.sixv_vertex_types(h) >= 0).all()


def test_cftp_samples_are_uniform_alternating_sign_matrices():
    n, runs = 3, 1400
    confs = po.sixv_enumerate(n)
    index = {c.tobytes(): k for k, c in enumerate(confs)}
    cnt = np.zeros(len(confs))
    for s in range(runs):
        h, _, _, ok = po.sixv_cftp(n, 2, s)
        assert ok
        cnt[index[h.tobytes()]] += 1
    e = runs / len(confs)
    chi2 = float(((cnt - e) ** 2 / e).sum())
    assert chi2 < 25.0, chi2  # 6 degrees of freedom
