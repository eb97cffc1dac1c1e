"""Step and sweep counts beyond what one call may ask for (2^40 colour steps;
2^35 batched sweeps; 2^38 six-vertex sweeps) are refused with RT_E_INVAL
before any schedule is sized from them, up to the largest int64, and the
caller's data stays as it was.  Without the bound, a count near 2^62 made the
phase list's byte size wrap to a few bytes.  The MLP's dataset row count is bounded
the same way (2^40).  Collected last so that a failure here cannot hide
other tests.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

HUGE = [(1 << 40) + 1, 1 << 62, (1 << 63) - 1]


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


def _refused(excinfo) -> None:
    from randomtilings_b200 import _capi

    assert excinfo.value.status == _capi.RT_E_INVAL
    assert "2^" in str(excinfo.value)


@pytest.mark.parametrize("steps", HUGE)
def test_walk_refuses_more_than_2_40_steps(rt, steps):
    from randomtilings_b200._capi import RtError

    t0 = np.array(golden("builders")["lozenge/hex13_5/min"], dtype=np.int32)
    t = t0.copy()
    tl = rt.LozengeTiler()
    with pytest.raises(RtError) as ei:
        tl.Walk(t, steps, 1)
    _refused(ei)
    assert np.array_equal(t, t0)
    # the handle still walks
    tl.Walk(t, 10, 1)
    tl.close()


def test_epoch_walk_refuses_a_total_above_2_40_steps(rt):
    from randomtilings_b200._capi import RtError

    t0 = np.array(golden("builders")["domino/aztec13/min"], dtype=np.int32)
    t = t0.copy()
    tl = rt.DominoTiler()
    with pytest.raises(RtError) as ei:
        tl.Walk(t, [1 << 39, 1 << 39, 1], [1, 2, 3])
    _refused(ei)
    assert np.array_equal(t, t0)
    tl.close()


@pytest.mark.parametrize("sweeps", [(1 << 38) + 1, (1 << 63) - 1])
def test_sixv_walk_and_cftp_refuse_more_than_2_38_sweeps(rt, sweeps):
    from randomtilings_b200._capi import RtError

    h0 = rt.SixVertexTiler.MinHeights(12)
    h = h0.copy()
    tl = rt.SixVertexTiler()
    with pytest.raises(RtError) as ei:
        tl.Walk(h, sweeps, 1)
    _refused(ei)
    assert np.array_equal(h, h0)
    with pytest.raises(RtError) as ei:
        tl.CFTP(12, first_sweeps=sweeps, master_seed=0)
    _refused(ei)
    tl.close()


@pytest.mark.parametrize("sweeps", [(1 << 35) + 1, (1 << 63) - 1])
def test_batch_refuses_more_than_2_35_sweeps(rt, sweeps):
    from randomtilings_b200._capi import RtError

    b = rt.Batch()
    with pytest.raises(RtError) as ei:
        b.run(sweeps)
    _refused(ei)
    with pytest.raises(RtError) as ei:
        b.set_sweeps_per_launch(sweeps)
    _refused(ei)
    b.close()


def test_walk_refuses_a_tiling_side_above_32767(rt):
    """The side is checked before the tiling is read, so a short buffer
    suffices; 32,769 is a multiple of 3, as a lozenge side must be."""
    from randomtilings_b200 import _capi

    buf = np.zeros(16, dtype=np.int32)
    tl = rt.LozengeTiler()
    st = tl._lib.rt_walk(tl._h, buf.ctypes.data, 32769, 10, 1)
    assert st == _capi.RT_E_INVAL
    assert "32767" in tl._lib.rt_last_error(tl._h).decode()
    assert not buf.any()
    tl.close()


def test_mlp_refuses_a_dataset_above_2_40_rows(rt):
    """A row count whose byte size would wrap is refused, and a handle
    without data refuses to train (it would have nothing to sample)."""
    from randomtilings_b200 import _capi
    from randomtilings_b200.mlp import CoordinateMLP

    m = CoordinateMLP()
    x = np.zeros((4, _capi.RT_MLP_IN), dtype=np.float32)
    t = np.zeros(4, dtype=np.float32)
    assert m._lib.rt_mlp_set_data(m._h, x.ctypes.data, t.ctypes.data, 1 << 62) == _capi.RT_E_INVAL
    loss = ctypes.c_float()
    assert m._lib.rt_mlp_train(m._h, 1, 16, 1e-3, 0, ctypes.byref(loss)) == _capi.RT_E_INVAL
    m.close()
