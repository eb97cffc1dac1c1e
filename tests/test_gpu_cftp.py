"""CFTP on the GPU (coupled max/min chains in one launch, device coalescence
test) against the oracle's CFTP composed from the restated epoch walk."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,first,schedule,seed", [
    (5, 128, "reference", 345903),   # the reference example's own settings
    (8, 128, "reference", 11),
    (13, 64, "doubling", 345903),
    (13, 32, "doubling", 7),
])
def test_cftp_matches_oracle(order, first, schedule, seed):
    import randomtilings_b200 as rt
    from randomtilings_b200 import _capi

    b = golden("builders")
    tmax, tmin = b[f"domino/aztec{order}/max"], b[f"domino/aztec{order}/min"]
    tl = rt.DominoTiler(kernel=_capi.RT_KERNEL_CFTP)
    sch = _capi.RT_CFTP_REFERENCE if schedule == "reference" else _capi.RT_CFTP_DOUBLING
    got, st = tl.CFTP(tmax, tmin, first_steps=first, schedule=sch, master_seed=seed, max_trials=20)
    want, trials, total, ok = po.cftp(tmax, tmin, first, seed, schedule, max_trials=20)
    assert st["coalesced"] and ok
    assert st["trials"] == trials and st["total_steps"] == total
    assert np.array_equal(got, want)


def test_cftp_sample_is_a_tiling_of_the_domain():
    import randomtilings_b200 as rt
    from randomtilings_b200 import _capi

    d = rt.DominoTiler.AztecDiamond(20)
    tmax, tmin = rt.DominoTiler.MaxTiling(d), rt.DominoTiler.MinTiling(d)
    tl = rt.DominoTiler(kernel=_capi.RT_KERNEL_CFTP)
    got, st = tl.CFTP(tmax, tmin, first_steps=256, master_seed=5, max_trials=20)
    assert st["coalesced"]
    # A valid domino tiling of the domain: its height function exists and maps back.
    h = rt.DominoTiler.TilingToHeightfunc(got, d)
    assert np.array_equal(rt.DominoTiler.HeightfuncToTiling(h, d), got)
    assert np.array_equal(rt.DominoTiler.TilingToDomain(got), rt.DominoTiler.TilingToDomain(tmin))


def test_cftp_rejects_the_non_monotone_kernel():
    import randomtilings_b200 as rt

    b = golden("builders")
    with pytest.raises(rt.RtError):
        rt.DominoTiler().CFTP(b["domino/aztec5/max"], b["domino/aztec5/min"])
