"""Pins the CPU restatement (oracle/rt_oracle.c) before anything trusts it.

Against: published known answers of the generators, the reference's own
code run on the CPU (tests/golden/*.npz, written by make_golden.py from
oracle/_ref), and -- where oracle/_ref is built here -- fresh reference runs
on random small cases.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import cases, golden
from oracle import pyoracle as po


class _Tiny(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("s0", "s1", "s2", "s3", "mat1", "mat2", "tmat")]


def test_tinymt32_known_answer():
    # The TinyMT32 check values for seed 1 and the TinyMT32J parameters
    # (tinymt32.out.txt of the TinyMT distribution); the reference exposes the
    # top 23 bits of each output through single01().
    s = _Tiny(0, 0, 0, 0, *po.TINYMT32J)
    lib = po.oracle()
    lib.orc_tinymt_init(ctypes.byref(s), 1)
    expect = [2545341989, 981918433, 3715302833, 2387538352, 3591001365]
    got = [lib.orc_tinymt_bits12(ctypes.byref(s)) & 0x7FFFFF for _ in expect]
    assert got == [e >> 9 for e in expect]


def test_mt19937_known_answer():
    # C++ [rand.predef]: the 10000th output of a default-seeded mt19937.
    out = np.zeros(10000, dtype=np.uint32)
    po.oracle().orc_mt19937_stream(5489, 10000, out.ctypes.data)
    assert int(out[-1]) == 4123659995


def test_minstd_rand0_known_answer():
    # C++ [rand.predef]: the 10000th output of a default-seeded minstd_rand0.
    out = np.zeros(10000, dtype=np.uint32)
    po.oracle().orc_minstd_raw_stream(1, 10000, out.ctypes.data)
    assert int(out[-1]) == 1043618065


@pytest.mark.parametrize("key", cases("walks", "domino/") + cases("walks", "domino_cftp/"))
def test_domino_walk_matches_reference(key):
    g = golden("walks")
    got = po.domino_walk(g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]),
                         cftp=key.startswith("domino_cftp"))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("key", cases("walks", "domino_epochs/"))
def test_domino_epoch_walk_matches_reference(key):
    g = golden("walks")
    got = po.domino_walk_epochs(g[f"{key}/start"], g[f"{key}/steps"], g[f"{key}/seeds"], cftp=True)
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("key", cases("walks", "lozenge/") + cases("walks", "qlozenge/"))
def test_lozenge_walk_matches_reference(key):
    # The reference's C++ build of qlozengekernel.cl compares q as a double.
    g = golden("walks")
    got = po.lozenge_walk(g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]),
                          qweight=key.startswith("qlozenge"), qcmp_double=True)
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("key", cases("walks", "recttri/"))
def test_recttri_walk_matches_reference(key):
    g = golden("walks")
    got = po.recttri_walk(g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.parametrize("steps", [10000, 20000])
def test_aztec100_matches_reference(steps):
    """Aztec n=100 from the minimal tiling, seed 42."""
    b, c = golden("builders"), golden("aztec100")
    got = po.domino_walk(b["domino/aztec100/min"], steps, 42)
    assert np.array_equal(got, c[f"cfg0/s{steps}/end"])


def test_q_comparison_modes_differ_at_one_draw_only():
    """qlozengekernel.cl:25 `q >= rd/.5` with the double literal q = 0.99 versus
    an fp32 device: over every 23-bit draw k the two accept differently only at
    k = 4152361 (2k * 2^-23 == float(0.99))."""
    k = np.arange(1 << 22, dtype=np.float64)
    x = (k * 2.0 ** -23 / 0.5).astype(np.float32).astype(np.float64)  # rd / .5, exact
    acc_double = 0.99 >= x
    acc_float = np.float64(np.float32(0.99)) >= x
    diff = np.nonzero(acc_double != acc_float)[0]
    assert diff.tolist() == [4152361]


@pytest.mark.skipif(not po.have_ref(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("seed", [1, 99, 123456789])
def test_fresh_reference_runs(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(6, 20))
    t = po.ref_build("domino_min", po.ref_build("domino_aztec", p0=n))
    steps = int(rng.integers(1, 400))
    for cftp, model in ((False, "domino"), (True, "domino_cftp")):
        r = po.RefTiler(model, t.size // 2).walk(t, steps, seed)
        assert np.array_equal(po.domino_walk(t, steps, seed, cftp=cftp), r)
    d = po.ref_build("lozenge_almost_hex", p0=int(rng.integers(3, 15)), p1=0)
    t = po.ref_build("lozenge_max", d)
    for qw, model in ((False, "lozenge"), (True, "qlozenge")):
        r = po.RefTiler(model, t.size).walk(t, steps, seed)
        assert np.array_equal(po.lozenge_walk(t, steps, seed, qweight=qw, qcmp_double=True), r)


@pytest.mark.skipif(not po.have_ref(), reason="oracle/_ref not built here")
def test_reference_serial_equals_threaded():
    """The oracle runs each NDRange serially or with OpenMP; the reference's
    kernels are race-free per launch, so both give the same tiling."""
    t = po.ref_build("domino_min", po.ref_build("domino_aztec", p0=20))
    a = po.RefTiler("domino", t.size // 2, threads=1).walk(t, 500, 3)
    b = po.RefTiler("domino", t.size // 2, threads=4).walk(t, 500, 3)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("key", cases("walks", "tridimer/"))
def test_tridimer_walk_matches_reference(key):
    g = golden("walks")
    got = po.tridimer_walk(g[f"{key}/start"], int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0]))
    assert np.array_equal(got, g[f"{key}/end"])


@pytest.mark.skipif(not po.have_ref(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("n,m,seed", [(12, 0, 1), (16, 4, 12345), (25, 7, -8)])
def test_tridimer_fresh_reference_runs(n, m, seed):
    t = po.ref_build("tridimer_ice_cream_cone", p0=n, p1=m)
    r = po.RefTiler("tridimer", t.size).walk(t, 2000, seed)
    assert np.array_equal(po.tridimer_walk(t, 2000, seed), r)


@pytest.mark.skipif(not po.have_ref(), reason="oracle/_ref not built here")
def test_cftp_composition_matches_reference_epoch_walks():
    """The oracle's CFTP (used by the GPU CFTP tests) against the same schedule
    driven through the reference's own epoch Walk."""
    b = golden("builders")
    tmax, tmin = b["domino/aztec5/max"], b["domino/aztec5/min"]
    got, trials, total, ok = po.cftp(tmax, tmin, 128, 345903, "reference")
    seeds = np.zeros(trials, dtype=np.uint32)
    po.oracle().orc_mt19937_stream(345903, trials, seeds.ctypes.data)
    steps = [256] * (trials - 1) + [128]  # newest epoch first
    sd = [int(s) for s in seeds[::-1]]
    rt = po.RefTiler("domino_cftp", tmax.size // 2)
    top, bot = rt.walk_epochs(tmax, steps, sd), rt.walk_epochs(tmin, steps, sd)
    assert ok and np.array_equal(top, bot) and np.array_equal(top, got)
