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
