"""Host builders of librt_b200.so against the reference's own outputs
(tests/golden/builders.npz, written from the reference by make_golden.py).
No GPU needed: these are the C++ host functions of the library."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

import randomtilings_b200 as rt

B = golden("builders")
D, L, R = rt.DominoTiler, rt.LozengeTiler, rt.RectTriangleTiler

AZTEC = [1, 2, 3, 5, 8, 13, 100]


@pytest.mark.parametrize("n", AZTEC)
def test_domino_aztec_domain_and_extremal_tilings(n):
    d = D.AztecDiamond(n)
    assert np.array_equal(d, B[f"domino/aztec{n}/domain"])
    assert np.array_equal(D.MinTiling(d), B[f"domino/aztec{n}/min"])
    assert np.array_equal(D.MaxTiling(d), B[f"domino/aztec{n}/max"])


@pytest.mark.parametrize("n", [k for k in AZTEC if k <= 13])
def test_domino_heights_vertices_domain(n):
    d = B[f"domino/aztec{n}/domain"]
    assert np.array_equal(D.DomainToVertices(d), B[f"domino/aztec{n}/vertices"])
    for which in ("min", "max"):
        t = B[f"domino/aztec{n}/{which}"]
        h = D.TilingToHeightfunc(t, d)
        assert np.array_equal(h, B[f"domino/aztec{n}/h{which}"])
        assert np.array_equal(D.HeightfuncToTiling(h, d), t)  # round trip
    assert np.array_equal(D.TilingToDomain(B[f"domino/aztec{n}/min"]), B[f"domino/aztec{n}/tiling_to_domain"])


@pytest.mark.parametrize("m,n", [(2, 2), (4, 6), (5, 8), (7, 7)])
def test_domino_rectangles(m, n):
    d = D.Rectangle(m, n)
    assert np.array_equal(d, B[f"domino/rect{m}x{n}/domain"])
    key = f"domino/rect{m}x{n}"
    if (m * n) % 2 == 0:
        assert np.array_equal(D.MinTiling(d), B[f"{key}/min"])
        assert np.array_equal(D.MaxTiling(d), B[f"{key}/max"])


@pytest.mark.parametrize("n,rem", [(4, (1,)), (6, (0, 2)), (7, (1, 3, 5))])
def test_domino_aztec_rectangle(n, rem):
    got = D.AztecRectangle(n, list(rem))
    assert np.array_equal(got, B[f"domino/aztecrect{n}_{'_'.join(map(str, rem))}/domain"])


HEX = [(2, 0), (4, 0), (4, 1), (10, 2), (13, 5), (20, 0)]


@pytest.mark.parametrize("n,m", HEX)
def test_lozenge_almost_hex(n, m):
    key = f"lozenge/hex{n}_{m}"
    d = L.AlmostHexDomain(n, m)
    assert np.array_equal(d, B[f"{key}/domain"])
    assert np.array_equal(L.DomainToVertices(d), B[f"{key}/vertices"])
    for which in ("min", "max"):
        t = getattr(L, f"{which.capitalize()}Tiling")(d)
        assert np.array_equal(t, B[f"{key}/{which}"])
        h = L.TilingToHeightfunc(t, d)
        assert np.array_equal(h, B[f"{key}/h{which}"])
        assert np.array_equal(L.HeightfuncToTiling(h, d), t)
    assert np.array_equal(L.TilingToDomain(B[f"{key}/min"]), B[f"{key}/tiling_to_domain"])
    assert np.array_equal(R.LozengeToRectTriangle(B[f"{key}/min"], d), B[f"{key}/recttri"])


@pytest.mark.parametrize("n", [1, 2, 3, 5, 6, 9, 20])
def test_recttri_hexagons(n):
    assert np.array_equal(R.maxHex(n), B[f"recttri/max_hex{n}"])
    assert np.array_equal(R.minHex(n), B[f"recttri/min_hex{n}"])


def test_not_tileable_is_an_error():
    d = D.Rectangle(3, 3)  # odd area
    with pytest.raises(rt.RtError):
        D.MinTiling(d)


T = rt.TriangleDimerTiler
CONES = [(6, 0), (5, 0), (8, 2), (10, 3), (12, 0)]


@pytest.mark.parametrize("n,m", CONES)
def test_tridimer_cone_and_derived_states(n, m):
    key = f"tridimer/cone{n}_{m}"
    t = T.IceCreamCone(n, m)
    assert np.array_equal(t, B[f"{key}/tiling"])
    assert np.array_equal(T.TilingToTriangleFlips(t), B[f"{key}/triangle_flips"])
    assert np.array_equal(T.TilingToButterflyFlips(t), B[f"{key}/butterfly_flips"])
    assert np.array_equal(T.TilingToVertices(t), B[f"{key}/vertices"])
    assert np.array_equal(T.TilingToDomain(t), B[f"{key}/domain"])
    for c in range(3):
        assert np.array_equal(T.DimerIndicator(t, c), B[f"{key}/dimer{c}"])


@pytest.mark.parametrize("k", [0, 1, 2])
def test_tridimer_test_butterfly(k):
    assert np.array_equal(T.TestButterfly(k), B[f"tridimer/butterfly{k}"])


def _macmahon(a: int, b: int, c: int) -> int:
    from fractions import Fraction

    p = Fraction(1)
    for i in range(1, a + 1):
        for j in range(1, b + 1):
            for k in range(1, c + 1):
                p *= Fraction(i + j + k - 1, i + j + k - 2)
    return int(p)


def test_lozenge_hexagon_generalises_almost_hex():
    import randomtilings_b200 as rt

    for n in (1, 2, 5, 13):
        assert np.array_equal(rt.LozengeTiler.Hexagon(n, n, n), rt.LozengeTiler.AlmostHexDomain(n, 0))


@pytest.mark.parametrize("a,b,c", [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2), (2, 2, 1), (1, 2, 3), (3, 1, 2),
                                   (2, 3, 2)])
def test_lozenge_hexagon_tilings(a, b, c):
    """Extremal tilings of the a x b x c hexagon tile exactly its domain, and
    chains started there reach MacMahon's number of tilings."""
    import randomtilings_b200 as rt
    from oracle import pyoracle as po

    d = rt.LozengeTiler.Hexagon(a, b, c)
    tmin, tmax = rt.LozengeTiler.MinTiling(d), rt.LozengeTiler.MaxTiling(d)
    assert np.array_equal(rt.LozengeTiler.TilingToDomain(tmin), d)
    assert np.array_equal(rt.LozengeTiler.TilingToDomain(tmax), d)
    seen = {po.walk_fast("lozenge", t0, 60, key).tobytes() for key in range(300) for t0 in (tmin, tmax)}
    assert len(seen) == _macmahon(a, b, c)
