"""The row-scan method of the device height functions (rt_height.cu), restated
in numpy and checked on the CPU against the host breadth-first
TilingToHeightfunc (byte-equal to the reference's): per row a prefix sum of
horizontal edge steps, rows tied together by one vertical edge each, the
first boundary vertex at 0.  Edge step: s when no tile crosses the edge,
-3s (dominoes) or -2s (lozenges) when one does."""
from __future__ import annotations

import functools

import numpy as np
import pytest

import randomtilings_b200 as rt
from oracle import pyoracle as po

INF = np.iinfo(np.int32).max


def scan_heights(model: int, t: np.ndarray, verts: np.ndarray) -> np.ndarray:
    n = verts.shape[0]
    t = t.reshape(n, n).astype(np.int64)
    dom = model == rt.RT_DOMINO
    out = np.full((n, n), INF, dtype=np.int64)
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    if dom:
        s = np.where((ii + jj) % 2 == 0, 1, -1)
        hstep = np.where(t & 8, -3 * s, s)
        sv = np.where((ii + jj) % 2 == 0, -1, 1)  # step of the edge (i, j) -> (i + 1, j)
        vstep = np.where(t & 2, -3 * sv, sv)
    else:
        hstep = np.where(t & 8, 2, -1)
        vstep = np.where(t & 32, -2, 1)
    rows = [np.flatnonzero(verts[i]) for i in range(n)]
    P = {}
    for i, js in enumerate(rows):
        if js.size == 0:
            continue
        lo, hi = js[0], js[-1]
        assert js.size == hi - lo + 1, "row is one run"
        P[i] = (lo, hi, np.concatenate([[0], np.cumsum(hstep[i, lo:hi])]))
    start = np.argwhere(verts == 2)[0]
    R = {}
    order = sorted(P)
    R[order[0]] = 0
    for i in order[1:]:
        lo, hi, p = P[i]
        plo, phi, pp = P[i - 1]
        c = (max(lo, plo) + min(hi, phi)) // 2  # any shared column whose edge touches the domain
        R[i] = R[i - 1] + pp[c - plo] + vstep[i - 1, c] - p[c - lo]
    i0, j0 = start
    shift = R[i0] + P[i0][2][j0 - P[i0][0]]
    for i, (lo, hi, p) in P.items():
        out[i, lo:hi + 1] = p + R[i] - shift
    return out.reshape(-1)


@functools.lru_cache(maxsize=None)
def _domino_cases():
    out = []
    for order in (3, 8, 17, 30):
        d = rt.DominoTiler.AztecDiamond(order)
        tmin = np.asarray(rt.DominoTiler.MinTiling(d), dtype=np.int32)
        tmax = np.asarray(rt.DominoTiler.MaxTiling(d), dtype=np.int32)
        out += [(d, tmin), (d, tmax), (d, po.domino_walk(tmin, 8 * order * order, 11 + order))]
    return out


@functools.lru_cache(maxsize=None)
def _lozenge_cases():
    out = []
    for dom in (rt.LozengeTiler.AlmostHexDomain(6, 0), rt.LozengeTiler.AlmostHexDomain(10, 3),
                rt.LozengeTiler.Hexagon(7, 12, 4), rt.LozengeTiler.Hexagon(15, 9, 11)):
        tmin = np.asarray(rt.LozengeTiler.MinTiling(dom), dtype=np.int32)
        tmax = np.asarray(rt.LozengeTiler.MaxTiling(dom), dtype=np.int32)
        out += [(dom, tmin), (dom, tmax), (dom, po.lozenge_walk(tmin, 3000, 5))]
    return out


@pytest.mark.parametrize("k", range(12))
def test_domino_row_scan_equals_bfs(k):
    d, t = _domino_cases()[k]
    verts = np.asarray(rt.DominoTiler.DomainToVertices(d), dtype=np.int32)
    n = int(round(verts.size ** 0.5))
    want = np.asarray(rt.DominoTiler.TilingToHeightfunc(t, d), dtype=np.int64)
    assert np.array_equal(scan_heights(rt.RT_DOMINO, t, verts.reshape(n, n)), want)


@pytest.mark.parametrize("k", range(12))
def test_lozenge_row_scan_equals_bfs(k):
    d, t = _lozenge_cases()[k]
    verts = np.asarray(rt.LozengeTiler.DomainToVertices(d), dtype=np.int32)
    n = int(round(verts.size ** 0.5))
    want = np.asarray(rt.LozengeTiler.TilingToHeightfunc(t, d), dtype=np.int64)
    assert np.array_equal(scan_heights(rt.RT_LOZENGE, t, verts.reshape(n, n)), want)
