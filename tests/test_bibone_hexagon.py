"""The bibone hexagon builder (rt_tridimer_hexagon; no reference
counterpart): a dimer cover of the triangular-lattice hexagon of side s less
its top-left corner, in the reference's triangle-dimer encoding.  Checked on
the CPU: the cover's edges, decoded from the tile states, meet every vertex
of the domain exactly once and no other; the reference's own reader
(TilingToVertices through oracle/_ref) sees the same vertices; the walks keep
them, and the reference's own walk equals the oracle's on it."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po


def hexagon_vertices(s: int, off: int = 3) -> set:
    return {(x + off, y + off) for x in range(2 * s + 1) for y in range(2 * s + 1)
            if s <= x + y <= 3 * s and (x, y) != (0, s)}


def decode_edges(t: np.ndarray) -> list:
    """Dimer edges from the tile states (TriangleDimerTiler.h:13-67): lozenge
    cells (even i, odd j) hold r, l, r, l and (odd i, odd j) h, l, h, l bits."""
    n = int(round(t.size ** 0.5))
    T = t.reshape(n, n)
    edges = set()
    for i in range(n):
        for j in range(1, n, 2):
            v = int(T[i, j])
            if i % 2 == 0:
                if v & 1:
                    edges.add(("r", i // 2 - 1, j // 2))
                if v & 2:
                    edges.add(("l", i // 2 - 1, j // 2 + 1))
                if v & 4:
                    edges.add(("r", i // 2, j // 2))
                if v & 8:
                    edges.add(("l", i // 2, j // 2))
            else:
                if v & 1:
                    edges.add(("h", i // 2, j // 2))
                if v & 4:
                    edges.add(("h", i // 2 + 1, j // 2))
                if v & 2:
                    edges.add(("l", i // 2, j // 2 + 1))
                if v & 8:
                    edges.add(("l", i // 2, j // 2))
    return sorted(edges)


def ends(kind, i, j):
    # h joins (i, j)-(i, j+1); l joins (i, j)-(i+1, j); r joins (i, j+1)-(i+1, j)
    return {"h": ((i, j), (i, j + 1)), "l": ((i, j), (i + 1, j)), "r": ((i, j + 1), (i + 1, j))}[kind]


@pytest.fixture(scope="module")
def td():
    import randomtilings_b200 as rt

    rt.load()
    return rt.TriangleDimerTiler


@pytest.mark.parametrize("s", [1, 2, 3, 4, 5, 8, 13, 64])
def test_cover_meets_every_vertex_once(td, s):
    t = np.asarray(td.BiboneHexagon(s))
    assert t.size == (4 * s + 16) ** 2
    deg = {}
    for e in decode_edges(t):
        for v in ends(*e):
            deg[v] = deg.get(v, 0) + 1
    assert set(deg) == hexagon_vertices(s)
    assert set(deg.values()) == {1}


@pytest.mark.parametrize("s", [2, 5, 64])
def test_vertices_as_the_library_and_the_reference_read_them(td, s):
    t = np.asarray(td.BiboneHexagon(s))
    v = np.asarray(td.TilingToVertices(t))
    m = int(round(v.size ** 0.5))
    got = {(i, j) for i in range(m) for j in range(m) if v[i * m + j]}
    assert got == hexagon_vertices(s)
    if po.have_ref():
        assert np.array_equal(v, po.ref_build("tridimer_vertices", t))


@pytest.mark.parametrize("s,seed", [(4, 1), (9, 42)])
def test_walks_keep_the_domain(td, s, seed):
    t = np.asarray(td.BiboneHexagon(s))
    v0 = np.asarray(td.TilingToVertices(t))
    w = po.tridimer_walk(t, 1500, seed)
    assert not np.array_equal(w, t)
    assert np.array_equal(np.asarray(td.TilingToVertices(w)), v0)
    f = po.walk_fast("tridimer", t, 1500, seed)
    assert np.array_equal(np.asarray(td.TilingToVertices(f)), v0)
    if po.have_ref():
        rt_ = po.RefTiler("tridimer", t.size)
        assert np.array_equal(rt_.walk(t, 1500, seed), w)
        rt_.close()
