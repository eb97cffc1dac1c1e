"""The oracle's bit-plane mode (oracle/rt_oracle.c plane_bit and the
bit-plane Rotates) on the CPU: walks keep the domain, the heat-bath rules are
monotone under shared bits (a walk from the maximal tiling stays above one
from the minimal tiling, vertex by vertex) and coalesce, and the bit layout
follows the documented Philox counters."""
from __future__ import annotations

import numpy as np
import pytest

import randomtilings_b200 as rt
from oracle import pyoracle as po


@pytest.mark.parametrize("name", ["domino", "domino_cftp", "lozenge"])
def test_walks_keep_the_domain(name):
    cls = rt.DominoTiler if name.startswith("domino") else rt.LozengeTiler
    d = cls.AztecDiamond(17) if cls is rt.DominoTiler else cls.Hexagon(9, 12, 7)
    t0 = np.asarray(cls.MinTiling(d), dtype=np.int32)
    t = po.walk_planes(name, t0, 200, 11)
    assert (t != t0).sum() > 20
    assert np.array_equal(cls.TilingToDomain(t), cls.TilingToDomain(t0))
    h = np.asarray(cls.TilingToHeightfunc(t, d))
    assert (h != np.iinfo(np.int32).max).sum() == (np.asarray(cls.TilingToHeightfunc(t0, d)) != np.iinfo(np.int32).max).sum()


@pytest.mark.parametrize("name", ["domino_cftp", "lozenge"])
def test_heat_bath_is_monotone(name):
    cls = rt.DominoTiler if name.startswith("domino") else rt.LozengeTiler
    d = cls.AztecDiamond(12) if cls is rt.DominoTiler else cls.Hexagon(7, 6, 8)
    top, bot = np.asarray(cls.MaxTiling(d), dtype=np.int32), np.asarray(cls.MinTiling(d), dtype=np.int32)
    inf = np.iinfo(np.int32).max
    for k in range(12):
        top, bot = po.walk_planes(name, top, 24, 100 + k), po.walk_planes(name, bot, 24, 100 + k)
        ht = np.asarray(cls.TilingToHeightfunc(top, d), dtype=np.int64)
        hb = np.asarray(cls.TilingToHeightfunc(bot, d), dtype=np.int64)
        m = ht != inf
        hi, lo = (ht, hb) if ht[m].sum() >= hb[m].sum() else (hb, ht)
        assert np.all(hi[m] >= lo[m]), k


def test_bit_layout():
    """A lozenge site flips 25 -> 38 exactly where its Philox bit is 1."""
    t = np.asarray(rt.LozengeTiler.MinTiling(rt.LozengeTiler.Hexagon(40, 40, 40)), dtype=np.int32)
    n = int(round(t.size ** 0.5))
    m = n // 3
    after = po.walk_planes("lozenge", t, 1, 7, chain=5)  # one step: colour 0 only
    ww = (m + 31) // 32
    qpr = (ww + 3) // 4
    for i in range(n):
        for jj in range(0, n, 3):
            j = jj + (i % 3)  # colour 0: (j - i) mod 3 == 0
            if j >= n or t[i * n + j] != 25:
                continue
            c = j // 3
            w = po.philox4x32_10([i * qpr + c // 128, 0, 0, 5], [7, 0])
            bit = (w[(c // 32) & 3] >> (c & 31)) & 1
            assert (after[i * n + j] == 38) == bool(bit), (i, j)
