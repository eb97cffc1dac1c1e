"""Validity checker for height functions (test helper): residues, the edge
rule, the boundary and the round trip through the reference's
HeightfuncToTiling / TilingToHeightfunc (rt_*_height_to_tiling here)."""
from __future__ import annotations

import numpy as np

INF = np.iinfo(np.int32).max
DOM_N = [(1, 0), (-1, 0), (0, 1), (0, -1)]
DOM_F = [((0, -1), (0, 0)), ((-1, -1), (-1, 0)), ((-1, 0), (0, 0)), ((-1, -1), (0, -1))]
LOZ_N = [(0, 1), (-1, 1), (-1, 0), (0, -1), (1, -1), (1, 0)]
LOZ_S = [-1, 1, -1, 1, -1, 1]
LOZ_F = [((0, 0), (-1, 1)), ((-1, 1), (-1, 0)), ((-1, 0), (-1, -1)), ((-1, -1), (0, -2)), ((0, -2), (0, -1)),
         ((0, -1), (0, 0))]


def check_height_function(model: str, domain, h, hmin, hmax) -> None:
    """Asserts h is a valid height function between hmin and hmax."""
    import randomtilings_b200 as rt

    d = np.asarray(domain).reshape(-1)
    h = np.asarray(h, dtype=np.int64).reshape(-1)
    lo = np.asarray(hmin, dtype=np.int64).reshape(-1)
    hi = np.asarray(hmax, dtype=np.int64).reshape(-1)
    n = int(round(h.size ** 0.5))
    m = n - 1
    dom = model == "domino"
    M = 4 if dom else 3
    inside = lo != INF
    assert np.array_equal(h == INF, ~inside)
    assert np.all((h[inside] - lo[inside]) % M == 0)
    assert np.all(lo[inside] <= h[inside]) and np.all(h[inside] <= hi[inside])

    def face(i, j):
        if dom:
            return 0 <= i < m and 0 <= j < m and d[i * m + j] != 0
        return 0 <= i < m and 0 <= j < 2 * m and d[i * 2 * m + j] != 0

    H = h.reshape(n, n)
    for i in range(n):
        for j in range(n):
            if H[i, j] == INF:
                continue
            for nb in range(4 if dom else 6):
                di, dj = (DOM_N if dom else LOZ_N)[nb]
                i2, j2 = i + di, j + dj
                if not (0 <= i2 < n and 0 <= j2 < n) or H[i2, j2] == INF:
                    continue
                (a, b), (c, e) = (DOM_F if dom else LOZ_F)[nb]
                ok = face(i + a, j + b) or face(i + c, j + e) if dom else face(i + a, 2 * j + b) or face(i + c, 2 * j + e)
                if not ok:
                    continue
                s = ((1 if nb > 1 else -1) * (1 if (i + j) % 2 == 0 else -1)) if dom else LOZ_S[nb]
                assert H[i2, j2] - H[i, j] in (s, -(M - 1) * s), (i, j, nb)
    cls = rt.DominoTiler if dom else rt.LozengeTiler
    t = cls.HeightfuncToTiling(h.astype(np.int32), d)
    assert np.array_equal(np.asarray(cls.TilingToHeightfunc(t, d)), h)
    assert np.array_equal(np.asarray(cls.TilingToDomain(t)), d)
