"""Bounded waits between the CTAs of a walk (no GPU fault, trap or hang):
a withheld halo row makes the neighbours' waits run out, the walk returns
RT_E_TIMEOUT, and the device stays usable; a walk longer than the wait
limit is unaffected, since each wait has its own clock."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["generic", "word"])
def test_withheld_row_times_out_and_device_recovers(monkeypatch, kernel):
    import randomtilings_b200 as rt

    t = golden("builders")["lozenge/hex20_0/min"]
    monkeypatch.setenv("RT_WALK_KERNEL", kernel)
    monkeypatch.setenv("RT_WAIT_TIMEOUT_MS", "100")
    monkeypatch.setenv("RT_TEST_DROP_PUBLISH", "7")
    tl = rt.LozengeTiler()
    a = np.array(t, dtype=np.int32)
    with pytest.raises(rt.RtError) as e:
        tl.Walk(a, 1000, 3)
    assert e.value.status == -5  # RT_E_TIMEOUT
    tl.close()
    monkeypatch.delenv("RT_TEST_DROP_PUBLISH")
    tl = rt.LozengeTiler()
    a = np.array(t, dtype=np.int32)
    tl.Walk(a, 1000, 3)
    assert np.array_equal(a, po.lozenge_walk(t, 1000, 3))


def test_walk_longer_than_the_wait_limit(monkeypatch):
    import randomtilings_b200 as rt

    monkeypatch.setenv("RT_WAIT_TIMEOUT_MS", "30")
    t = golden("builders")["lozenge/hex20_0/min"]
    tl = rt.LozengeTiler(rng=rt.RT_RNG_PHILOX)
    a = np.array(t, dtype=np.int32)
    tl.Walk(a, 150000, 9)  # about a third of a second
    assert np.array_equal(a, po.walk_fast("lozenge", t, 150000, 9))
