"""The update rules of the device extremal-tiling relaxation
(csrc/rt_extremal.cu), restated in numpy: their fixpoint from the boundary
heights equals the height functions of the host MaxTiling / MinTiling
(Thurston's flood, DominoTiler.cpp:214-399, LozengeTiler.cpp:140-318), which
are byte-equal to the reference's.  CPU only; the kernels themselves are
checked against the host builders in test_gpu_extremal.py."""
from __future__ import annotations

import numpy as np
import pytest

INF = np.iinfo(np.int32).max
BIG = 0x3FFFFFFF


def _relax_fixpoint(model, kind, boundary_h):
    """Jacobi iteration of the kernel's rules to their fixpoint."""
    n = kind.shape[0]
    hx = np.full((n + 2, n + 2), BIG, np.int64)
    hn = np.full((n + 2, n + 2), -BIG, np.int64)
    b = kind == 2
    hx[1:-1, 1:-1][b] = boundary_h[b]
    hn[1:-1, 1:-1][b] = boundary_h[b]
    i, j = np.indices((n, n))
    even = ((i + j) & 1) == 0
    inner = kind == 1

    def up(a):
        return a[:-2, 1:-1]

    def dn(a):
        return a[2:, 1:-1]

    def lf(a):
        return a[1:-1, :-2]

    def rg(a):
        return a[1:-1, 2:]

    for _ in range(10 * n):
        x, y = hx[1:-1, 1:-1], hn[1:-1, 1:-1]
        if model == 0:
            # even vertex: +1 horizontally, -1 vertically (DominoTiler.cpp:221-231); odd: the reverse
            vx = np.where(even, np.minimum(up(hx), dn(hx)), np.minimum(lf(hx), rg(hx))) + 1
            vn = np.where(even, np.maximum(lf(hn), rg(hn)), np.maximum(up(hn), dn(hn))) - 1
        else:
            # edges (0,+1), (-1,0), (+1,-1) step -1 from the vertex; the opposite three +1
            vx = np.minimum(np.minimum(rg(hx), up(hx)), hx[2:, :-2]) + 1
            vn = np.maximum(np.maximum(hn[:-2, 2:], lf(hn)), dn(hn)) - 1
        nx = np.where(inner, np.minimum(x, vx), x)
        ny = np.where(inner, np.maximum(y, vn), y)
        if np.array_equal(nx, x) and np.array_equal(ny, y):
            break
        hx[1:-1, 1:-1], hn[1:-1, 1:-1] = nx, ny
    x, y = hx[1:-1, 1:-1].copy(), hn[1:-1, 1:-1].copy()
    x[(kind == 0) | (x >= BIG)] = INF
    y[(kind == 0) | (y <= -BIG)] = INF
    return x, y


def _young(rows):
    """Domino domain of a Young diagram with even row lengths (tileable)."""
    m = max(len(rows), max(rows)) + 2
    d = np.zeros((m, m), np.int32)
    for r, length in enumerate(rows):
        d[r + 1, 1:1 + length] = 1
    return d.reshape(-1)


def _domains():
    import randomtilings_b200 as rt
    from randomtilings_b200 import builders

    out = [(0, rt.DominoTiler.AztecDiamond(k)) for k in (1, 2, 3, 8, 13, 24)]
    out += [(0, builders.call("rt_domino_rectangle", r, c)) for r, c in ((2, 2), (4, 6), (7, 8))]
    out += [(0, builders.aztec_rectangle(6, [1, 3])), (0, _young([8, 8, 6, 4, 4, 2]))]
    out += [(1, rt.LozengeTiler.Hexagon(a, b, c)) for a, b, c in ((1, 1, 1), (2, 3, 4), (7, 3, 9), (12, 12, 12))]
    out += [(1, rt.LozengeTiler.AlmostHexDomain(k, c)) for k, c in ((10, 2), (6, 0))]
    return out


@pytest.mark.parametrize("case", range(17))
def test_relaxation_fixpoint_is_the_flood(case):
    import randomtilings_b200 as rt
    from randomtilings_b200 import builders

    model, d = _domains()[case]
    cls = rt.DominoTiler if model == 0 else rt.LozengeTiler
    kind = builders.call("rt_domino_domain_to_vertices" if model == 0 else "rt_lozenge_domain_to_vertices", d)
    n = int(round(len(kind) ** 0.5))
    kind = kind.reshape(n, n)
    hmax = np.asarray(cls.TilingToHeightfunc(cls.MaxTiling(d), d)).reshape(n, n)
    hmin = np.asarray(cls.TilingToHeightfunc(cls.MinTiling(d), d)).reshape(n, n)
    assert np.array_equal(hmax[kind == 2], hmin[kind == 2])  # the boundary is fixed
    x, y = _relax_fixpoint(model, kind, hmax)
    assert np.array_equal(x, hmax)
    assert np.array_equal(y, hmin)


def test_case_count():
    assert len(_domains()) == 17
