"""GPU parity of the bit-exact walks, through the C ABI (librt_b200.so).

Every case compares the CUDA result with the oracle on the same input:
the golden reference outputs (tests/golden/walks.npz, aztec100.npz) and the
C restatement on further seeds / sizes.  Integer tilings: bit-exact.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cases, golden
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


def _walk(tiler, t, steps, seed):
    a = np.array(t, dtype=np.int32)
    tiler.Walk(a, steps, seed)
    return a


@pytest.mark.parametrize("key", cases("walks", "domino/") + cases("walks", "domino_cftp/"))
def test_domino_golden(rt, key):
    g = golden("walks")
    kernel = 1 if key.startswith("domino_cftp") else 0
    tl = rt.DominoTiler(kernel=kernel)
    got = _walk(tl, g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("key", cases("walks", "domino_epochs/"))
def test_domino_epochs_golden(rt, key):
    g = golden("walks")
    tl = rt.DominoTiler(kernel=1)
    a = np.array(g[f"{key}/start"], dtype=np.int32)
    tl.Walk(a, list(g[f"{key}/steps"]), list(g[f"{key}/seeds"]))
    assert np.array_equal(a, g[f"{key}/end"])


@pytest.mark.parametrize("key", cases("walks", "lozenge/"))
def test_lozenge_golden(rt, key):
    g = golden("walks")
    tl = rt.LozengeTiler()
    got = _walk(tl, g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("key", cases("walks", "qlozenge/"))
def test_qlozenge_golden_double_compare(rt, key):
    g = golden("walks")
    tl = rt.LozengeTiler(kernel=2, qcmp=1)
    got = _walk(tl, g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("key", cases("walks", "recttri/"))
def test_recttri_golden(rt, key):
    g = golden("walks")
    tl = rt.RectTriangleTiler()
    got = _walk(tl, g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("steps", [10000, 20000])
def test_aztec100(rt, steps):
    """Aztec diamond n=100, seed 42: bit-exact with the reference's kernels run on the host CPU."""
    b, c = golden("builders"), golden("aztec100")
    tl = rt.DominoTiler()
    got = _walk(tl, b["domino/aztec100/min"], steps, 42)
    assert np.array_equal(got, c[f"cfg0/s{steps}/end"])


@pytest.mark.parametrize("seed", [0, 17, 2**31 + 5, -123])
@pytest.mark.parametrize("qcmp", [0, 1])
def test_qlozenge_vs_restatement(rt, seed, qcmp):
    b = golden("builders")
    t = b["lozenge/hex20_0/min"]
    tl = rt.LozengeTiler(kernel=2, qcmp=qcmp, q=0.99)
    got = _walk(tl, t, 3000, seed)
    assert np.array_equal(got, po.lozenge_walk(t, 3000, seed, qweight=True, q=0.99, qcmp_double=bool(qcmp)))


@pytest.mark.parametrize("q", [0.5, 1.0, 1.7])
def test_qlozenge_other_q(rt, q):
    t = golden("builders")["lozenge/hex13_5/max"]
    for qcmp in (0, 1):
        tl = rt.LozengeTiler(kernel=2, qcmp=qcmp, q=q)
        got = _walk(tl, t, 2000, 77)
        assert np.array_equal(got, po.lozenge_walk(t, 2000, 77, qweight=True, q=q, qcmp_double=bool(qcmp)))


def test_recttri_nonunit_weights(rt):
    w = np.array([0.0, 1.0, 2.0, 0.5, 1.5, 0.7, 1.1, 1.5, 0.7, 1.1, 0.3, 3.0, 1.0, 0.3, 3.0, 1.0], dtype=np.float32)
    t = golden("builders")["recttri/slope_hex9"]
    tl = rt.RectTriangleTiler(weights=w)
    got = _walk(tl, t, 3000, 5)
    assert np.array_equal(got, po.recttri_walk(t, 3000, 5, weights=w))


def test_loaded_parameter_table(rt, tmp_path):
    """LoadTinyMT with a non-uniform table (file layout of file_reader.cpp)."""
    t = golden("builders")["domino/aztec13/min"]
    n = int(round(t.size ** 0.5))
    rng = np.random.default_rng(3)
    tab = rng.integers(0, 2**32, size=(n * n // 2, 3), dtype=np.uint64).astype(np.uint32)
    path = tmp_path / "tinymt.txt"
    with open(path, "w") as f:
        f.write("# synthetic table\n")
        for i, (a, b, c) in enumerate(tab):
            f.write(f"x,{i},127,{a:x},{b:x},{c:x},0,0\n")
    tl = rt.DominoTiler()
    tl.LoadTinyMT(str(path), n * n // 2)
    got = _walk(tl, t, 500, 11)
    assert np.array_equal(got, po.domino_walk(t, 500, 11, params=tab))


def test_large_lozenge_run_matches_restatement(rt):
    """A lattice spread over hundreds of CTAs (neighbour waits on every row band)."""
    t = golden("builders")["lozenge/hex20_0/min"]
    tl = rt.LozengeTiler()
    got = _walk(tl, t, 5000, 2024)
    assert np.array_equal(got, po.lozenge_walk(t, 5000, 2024))


def test_zero_steps_is_identity(rt):
    t = golden("builders")["domino/aztec8/min"]
    tl = rt.DominoTiler()
    assert np.array_equal(_walk(tl, t, 0, 1), t)


def test_bad_sizes_are_rejected(rt):
    tl = rt.DominoTiler()
    with pytest.raises(rt.RtError):
        tl.Walk(np.zeros(7 * 7, dtype=np.int32), 10, 1)
    tl = rt.LozengeTiler()
    with pytest.raises(rt.RtError):
        tl.Walk(np.zeros(10 * 10, dtype=np.int32), 10, 1)


@pytest.mark.parametrize("key", cases("walks", "tridimer/"))
def test_tridimer_golden(rt, key):
    g = golden("walks")
    tl = rt.TriangleDimerTiler()
    got = _walk(tl, g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("n,m,seed", [(12, 0, 1), (20, 0, 99), (25, 7, -8), (40, 10, 2024)])
def test_tridimer_vs_restatement(rt, n, m, seed):
    t = rt.TriangleDimerTiler.IceCreamCone(n, m)
    tl = rt.TriangleDimerTiler()
    got = _walk(tl, t, 3000, seed)
    assert np.array_equal(got, po.tridimer_walk(t, 3000, seed))


@pytest.mark.parametrize("k", [0, 1, 2])
def test_tridimer_single_butterflies(rt, k):
    t = rt.TriangleDimerTiler.TestButterfly(k)
    got = _walk(rt.TriangleDimerTiler(), t, 500, 5)
    assert np.array_equal(got, po.tridimer_walk(t, 500, 5))
