"""Device height functions (include/rt_b200_height.h) against the host
TilingToHeightfunc (byte-equal to the reference's), on tilings uploaded to the
device, on a Tiler's own device tiling after a walk, and on batch chains."""
from __future__ import annotations

import numpy as np
import pytest

import randomtilings_b200 as rt
from randomtilings_b200.heights import HeightPlan
from test_height_scan import _domino_cases, _lozenge_cases

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("model,k", [(rt.RT_DOMINO, k) for k in range(12)] + [(rt.RT_LOZENGE, k) for k in range(12)])
def test_device_heights_equal_host(model, k):
    import torch

    cls = rt.DominoTiler if model == rt.RT_DOMINO else rt.LozengeTiler
    d, t = (_domino_cases() if model == rt.RT_DOMINO else _lozenge_cases())[k]
    want = np.asarray(cls.TilingToHeightfunc(t, d), dtype=np.int32)
    plan = HeightPlan(model, d)
    assert plan.n * plan.n == t.size
    dt = _dev(np.asarray(t, dtype=np.int32))
    dh = torch.empty_like(dt)
    plan.heights(dt.data_ptr(), dh.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(dh.cpu().numpy(), want)
    inside = want != np.iinfo(np.int32).max
    # running sums: two accumulations = 2 h inside the domain, untouched outside
    s = torch.full((t.size,), 7, dtype=torch.int64, device="cuda")
    plan.accumulate(dt.data_ptr(), s.data_ptr())
    plan.accumulate(dt.data_ptr(), s.data_ptr())
    torch.cuda.synchronize()
    sv = s.cpu().numpy()
    assert np.array_equal(sv[inside], 7 + 2 * want[inside].astype(np.int64))
    assert np.all(sv[~inside] == 7)
    # mean |h - ref| over domain vertices
    ref = np.where(inside, want.astype(np.float32) + 0.25, 0).astype(np.float32)
    ref[np.flatnonzero(inside)[::3]] -= 1.0  # every third vertex: |h - ref| = 0.75
    e = plan.error(dt.data_ptr(), _dev(ref).data_ptr())
    want_e = np.abs(want[inside].astype(np.float64) - ref[inside]).mean()
    assert abs(e - want_e) < 1e-9 and plan.vertices == int(inside.sum())
    plan.close()


def test_rejects_unsupported_domains():
    # a domino domain with a row split in two runs (two squares joined below)
    d = np.zeros((6, 6), dtype=np.int32)
    d[0:2, 0:2] = 1
    d[0:2, 4:6] = 1
    d[2:4, 0:6] = 1
    with pytest.raises(rt.RtError):
        HeightPlan(rt.RT_DOMINO, d.reshape(-1))


@pytest.mark.parametrize("model", [rt.RT_DOMINO, rt.RT_LOZENGE])
def test_tiler_device_tiling_after_a_walk(model):
    import torch

    cls = rt.DominoTiler if model == rt.RT_DOMINO else rt.LozengeTiler
    d = cls.AztecDiamond(40) if model == rt.RT_DOMINO else cls.Hexagon(20, 31, 17)
    t0 = np.asarray(cls.MinTiling(d), dtype=np.int32)
    tl = cls(rng=rt.RT_RNG_PHILOX)
    tl.upload(t0)
    tl.run(3000, 9)
    ptr = tl.device_tiling()
    plan = HeightPlan(model, d)
    dh = torch.empty(t0.size, dtype=torch.int32, device="cuda")
    tl.synchronize()
    plan.heights(ptr, dh.data_ptr())
    torch.cuda.synchronize()
    host = np.zeros_like(t0)
    tl.download(host)
    assert not np.array_equal(host, t0)
    assert np.array_equal(dh.cpu().numpy(), np.asarray(cls.TilingToHeightfunc(host, d), dtype=np.int32))
    tl.close()


def test_batch_device_tiling_equals_download():
    import torch

    bt = rt.Batch()
    d1 = rt.DominoTiler.AztecDiamond(23)
    d2 = rt.LozengeTiler.Hexagon(9, 14, 11)
    i1 = bt.add(rt.RT_DOMINO, rt.DominoTiler.MinTiling(d1), key=3)
    i2 = bt.add(rt.RT_LOZENGE, rt.LozengeTiler.MinTiling(d2), key=4)
    bt.run(50)
    for idx in (i1, i2):
        host = bt.download(idx)
        dt = torch.zeros(host.size, dtype=torch.int32, device="cuda")
        bt.device_tiling(idx, dt.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(dt.cpu().numpy(), host)
    bt.close()
