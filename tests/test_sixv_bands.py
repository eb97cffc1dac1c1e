"""The six-vertex band kernel's halo protocol, rebuilt on the CPU from the
restatement.  Each band of face rows walks on its own copy of the heights
and sees its neighbours' edge rows only when the kernel exchanges them:
before every even colour step, with the rows the neighbours held after the
odd step before it.  That must give the whole-lattice walk for every band
height, because steps 2t and 2t + 1 update rows of one parity and the halo
rows they read have the other.  Exchanging before every step must agree
too; exchanging only before every fourth step, a planted mistake, must
not.  No GPU."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po


def band_walk(h0: np.ndarray, sweeps: int, key: int, rpc: int, exchange) -> np.ndarray:
    """The walk as bands of `rpc` face rows compute it, each on its own copy,
    halo rows refreshed before step s wherever exchange(s) holds."""
    a0 = np.array(h0, dtype=np.int32).reshape(-1)
    S = int(round(a0.size ** 0.5))
    bands = [(r0, min(S, r0 + rpc)) for r0 in range(0, S, rpc)]
    copies = [a0.copy() for _ in bands]
    for s in range(4 * sweeps):
        if s > 0 and exchange(s):
            # the rows each neighbour owns, as they stood after step s - 1
            for b, (r0, r1) in enumerate(bands):
                if b > 0:
                    copies[b][(r0 - 1) * S:r0 * S] = copies[b - 1][(r0 - 1) * S:r0 * S]
                if b + 1 < len(bands):
                    copies[b][r1 * S:(r1 + 1) * S] = copies[b + 1][r1 * S:(r1 + 1) * S]
        for b, (r0, r1) in enumerate(bands):
            po.sixv_step_rows(copies[b], s, key, r0, r1)
    out = np.empty_like(a0)
    for b, (r0, r1) in enumerate(bands):
        out[r0 * S:r1 * S] = copies[b][r0 * S:r1 * S]
    return out


def _kernel_rule(s: int) -> bool:
    return s % 2 == 0


@pytest.mark.parametrize("n", [9, 23, 40])
@pytest.mark.parametrize("rpc", [1, 2, 3, 4, 7])
def test_exchange_before_even_steps_gives_the_walk(n, rpc):
    for start in po.sixv_dwbc(n):
        want = po.sixv_walk(start, 24, 0xB17E5)
        got = band_walk(start, 24, 0xB17E5, rpc, _kernel_rule)
        assert np.array_equal(got, want)


def test_exchange_before_every_step_gives_the_walk():
    start = po.sixv_dwbc(23)[0]
    assert np.array_equal(band_walk(start, 24, 7, 3, lambda s: True), po.sixv_walk(start, 24, 7))


@pytest.mark.parametrize("rpc", [2, 3, 7])
def test_exchange_every_fourth_step_differs(rpc):
    """The planted mistake: halo rows refreshed only before steps 4t miss
    the rows the neighbours changed at steps 4t + 2 and 4t + 3."""
    start = po.sixv_dwbc(40)[0]
    assert not np.array_equal(band_walk(start, 24, 0xB17E5, rpc, lambda s: s % 4 == 0),
                              po.sixv_walk(start, 24, 0xB17E5))
