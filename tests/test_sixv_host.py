"""Host side of the six-vertex API (include/rt_b200_sixv.h), no GPU: the
domain-wall extremes, validity check, alternating-sign matrix and vertex
types agree with the restatement on every state of small grids."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po


@pytest.fixture(scope="module")
def sv():
    import randomtilings_b200 as rt

    rt.load()
    return rt.SixVertexTiler


@pytest.mark.parametrize("n", [1, 2, 5, 17])
def test_extremes(sv, n):
    lo, hi = po.sixv_dwbc(n)
    assert np.array_equal(sv.MinHeights(n), lo) and np.array_equal(sv.MaxHeights(n), hi)
    assert sv.IsValid(lo) and sv.IsValid(hi)


@pytest.mark.parametrize("n", [3, 4])
def test_every_state(sv, n):
    for h in po.sixv_enumerate(n):
        assert sv.IsValid(h)
        assert np.array_equal(sv.VertexTypes(h), po.sixv_vertex_types(h))
        a = sv.HeightsToASM(h)
        assert set(np.unique(a)) <= {-1, 0, 1}
        assert (a.sum(axis=0) == 1).all() and (a.sum(axis=1) == 1).all()
        # partial sums along rows and columns alternate: 0 or 1
        assert ((np.cumsum(a, axis=0) >= 0) & (np.cumsum(a, axis=0) <= 1)).all()
        assert ((np.cumsum(a, axis=1) >= 0) & (np.cumsum(a, axis=1) <= 1)).all()
        # the c-type vertices are exactly the non-zero entries
        assert np.array_equal(sv.VertexTypes(h) >= 4, a != 0)


def test_invalid_states_are_rejected(sv):
    h = sv.MinHeights(4).copy()
    h[6] = 1  # interior face (1, 1) at the wrong parity
    assert not sv.IsValid(h)
    h = sv.MinHeights(4).copy()
    h[0] = 1  # boundary
    assert not sv.IsValid(h)


def _exact_check(h: np.ndarray) -> bool:
    """The definition, in exact integers: boundary rows and columns 0..n as
    domain-wall conditions fix them, and every edge joining heights that
    differ by exactly 1."""
    n1 = int(round(h.size ** 0.5))
    n = n1 - 1
    a = h.reshape(n1, n1).astype(np.int64)
    k = np.arange(n1)
    if not (np.array_equal(a[0], k) and np.array_equal(a[:, 0], k) and np.array_equal(a[n], n - k)
            and np.array_equal(a[:, n], n - k)):
        return False
    return bool((np.abs(np.diff(a, axis=0)) == 1).all() and (np.abs(np.diff(a, axis=1)) == 1).all())


@pytest.mark.parametrize("n", [5, 40, 301])
def test_check_agrees_with_the_definition_on_damaged_walks(sv, n):
    """States of a real walk, then single faces set to values that break an
    edge by any amount, including the int32 extremes next to each other
    (whose difference is 1 modulo 2^32), and rows swapped."""
    rng = np.random.default_rng(n)
    h0 = po.sixv_walk(po.sixv_dwbc(n)[0], 30, 11)
    assert sv.IsValid(h0) and _exact_check(h0)
    lo, hi = np.iinfo(np.int32).min, np.iinfo(np.int32).max
    for trial in range(60):
        h = h0.copy().reshape(n + 1, n + 1)
        i, j = (int(v) for v in rng.integers(0, n + 1, size=2))
        kind = trial % 6
        if kind == 0:
            h[i, j] += 2
        elif kind == 1:
            h[i, j] = lo
        elif kind == 2:
            h[i, j] = hi
        elif kind == 3:
            h[i, j] = lo
            h[i, (j + 1) % (n + 1)] = hi
        elif kind == 4:
            h[[i, (i + 1) % (n + 1)]] = h[[(i + 1) % (n + 1), i]]
        else:
            h[i, j] -= 2 ** 31 - 1  # far from its neighbours, still an int32
        h = h.reshape(-1)
        assert sv.IsValid(h) == _exact_check(h), (trial, i, j)
