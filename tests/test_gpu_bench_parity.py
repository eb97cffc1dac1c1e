"""GPU parity of the bench's own workloads, at their full sizes, through the C ABI.

The bench walks the a=b=c=500 hexagon (LozengeTiler::AlmostHexDomain(500, 0)
-> MinTiling, a 1008 x 1008 tiling, 338,688 attempts per colour step) as 20
Walk calls of 3,000 colour steps with seeds 42..61, each continuing from the
last (20,000 sweeps), on the default handle: the word kernel on the bench's
grid.  tests/golden/bench_parity.json holds the SHA-256 of the reference's own
result after every call (LozengeTiler::Walk and lozengekernel.cl run on the
host), of the q = 0.99 int32 walk in both comparisons (qlozengekernel.cl built
in double and in single precision) from the uniform walk's end to a step
count where they part, and of the fast and bit-plane modes (the oracle's
replays, no reference counterpart), beside the Aztec diamond of order 2000.
Integer tilings: bit-exact, compared by digest.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, cases, golden

pytestmark = pytest.mark.gpu

SEGMENT = 3000


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


@pytest.fixture(scope="module")
def want():
    with open(os.path.join(GOLDEN, "bench_parity.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def hex500(rt, want):
    t = np.asarray(rt.LozengeTiler.MinTiling(rt.LozengeTiler.AlmostHexDomain(500, 0)), dtype=np.int32)
    assert digest(t) == want["hex500/start"]
    return t


@pytest.fixture(scope="module")
def aztec2000(rt, want):
    t = np.asarray(rt.DominoTiler.MinTiling(rt.DominoTiler.AztecDiamond(2000)), dtype=np.int32)
    assert digest(t) == want["aztec2000/start"]
    return t


@pytest.fixture(scope="module")
def hex500_walked(rt, want, hex500):
    """The bench's `value` leg: the lattice stays on the device between the 20
    calls (rt_upload once, rt_run per call); each call's result is read back
    and compared.  Returns the final tiling."""
    tl = rt.LozengeTiler()
    tl.upload(hex500)
    out = np.empty_like(hex500)
    for k in range(20):
        tl.run(SEGMENT, 42 + k)
        tl.download(out)
        assert digest(out) == want[f"hex500/uniform/segment{k}"], f"call {k}"
    tl.close()
    return out


def test_hex500_bench_walk_device_resident(hex500_walked, want):
    assert digest(hex500_walked) == want["hex500/uniform/segment19"]


def test_hex500_bench_walk_host_buffers(rt, want, hex500):
    """The bench's `e2e` leg: rt_walk with the host tiling every call."""
    tl = rt.LozengeTiler()
    a = hex500.copy()
    for k in range(20):
        tl.Walk(a, SEGMENT, 42 + k)
        assert digest(a) == want[f"hex500/uniform/segment{k}"], f"call {k}"
    tl.close()


def test_hex500_single_walk(rt, want, hex500):
    a = hex500.copy()
    rt.LozengeTiler().Walk(a, 600, 42)
    assert digest(a) == want["hex500/uniform/s42/600"]


@pytest.mark.parametrize("qcmp,name", [(0, "qf32"), (1, "qdouble")])
def test_hex500_q(rt, want, hex500_walked, qcmp, name):
    """q = 0.99 on int32 storage from the uniform walk's final tiling, to a
    step count at which the float32 and the double comparison of
    qlozengekernel.cl:25 give different tilings."""
    assert want["hex500/q/start"] == "hex500/uniform/segment19"
    a = hex500_walked.copy()
    rt.LozengeTiler(kernel=2, q=0.99, qcmp=qcmp).Walk(a, int(want["hex500/q/steps"]), int(want["hex500/q/seed"]))
    assert digest(a) == want[f"hex500/{name}"]


def test_hex500_q_modes_differ(want):
    assert want["hex500/qf32"] != want["hex500/qdouble"]


@pytest.mark.parametrize("mode", ["fast", "planes"])
def test_hex500_counter_modes(rt, want, hex500, mode):
    rng = rt.RT_RNG_PHILOX if mode == "fast" else rt.RT_RNG_PLANES
    a = hex500.copy()
    rt.LozengeTiler(rng=rng).Walk(a, 600, 42)
    assert digest(a) == want[f"hex500/{mode}/k42/600"]


@pytest.mark.parametrize("mode,kernel", [("fast", 0), ("planes", 0), ("planes_hb", 1)])
def test_aztec2000_counter_modes(rt, want, aztec2000, mode, kernel):
    rng = rt.RT_RNG_PHILOX if mode == "fast" else rt.RT_RNG_PLANES
    a = aztec2000.copy()
    rt.DominoTiler(kernel=kernel, rng=rng).Walk(a, 100, 42)
    assert digest(a) == want[f"aztec2000/{mode}/k42/100"]


@pytest.mark.parametrize("key", cases("qlozenge_f32", "qlozenge_f32/"))
def test_qlozenge_float32_golden(rt, key):
    """qlozengekernel.cl built with single-precision arithmetic (an fp32-only
    OpenCL device) against the float32 comparison, the double build against
    the double comparison; the a=b=c=40 cases stop right after a draw at
    which the two part."""
    g = golden("qlozenge_f32")
    steps, seed = int(g[f"{key}/steps"][0]), int(g[f"{key}/seed"][0])
    for qcmp, end in ((0, "end"), (1, "end_double")):
        a = np.array(g[f"{key}/start"], dtype=np.int32)
        rt.LozengeTiler(kernel=2, q=0.99, qcmp=qcmp).Walk(a, steps, seed)
        assert np.array_equal(a, g[f"{key}/{end}"]), (key, end)


@pytest.mark.parametrize("steps", [10000, 20000])
def test_aztec100_heights_on_device(rt, steps):
    """The Aztec n=100 walk from seed 42: the height function of the final
    tiling (device TilingToHeightfunc) equals the reference's."""
    import torch

    from randomtilings_b200.heights import HeightPlan

    b, c = golden("builders"), golden("aztec100")
    end = c[f"cfg0/s{steps}/end"]
    plan = HeightPlan(rt.RT_DOMINO, b["domino/aztec100/domain"])
    dt = torch.from_numpy(np.ascontiguousarray(end, dtype=np.int32)).cuda()
    dh = torch.empty_like(dt)
    plan.heights(dt.data_ptr(), dh.data_ptr())
    torch.cuda.synchronize()
    plan.close()
    assert np.array_equal(dh.cpu().numpy(), c[f"cfg0/s{steps}/height"])
