"""The fast mode's CPU restatement (oracle/rt_oracle.c, *_fast): its
generator against the published Philox4x32-10 known answers, and its chains
against the exact stationary law on domains small enough to enumerate."""
from __future__ import annotations

from collections import Counter

import numpy as np
import pytest
from scipy import stats

from conftest import golden
from oracle import pyoracle as po


# Known-answer vectors of Philox4x32-10 published with the Random123 library
# (counter, key) -> output.
KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert po.philox4x32_10(ctr, key) == want


# The statistical tests are deterministic (fixed keys and seeds); a law that
# is right fails them with probability 1e-4 (the p-value threshold).
P_MIN = 1e-4


def _uniform_pvalue(samples: list[bytes], n_states: int) -> float:
    counts = np.array(list(Counter(samples).values()))
    assert len(counts) == n_states
    return stats.chisquare(counts).pvalue


def test_fast_domino_chains_are_uniform_on_aztec2():
    """Aztec diamond of order 2 has 2^3 = 8 domino tilings; chain ends with
    independent keys must be uniform over them (both flip kernels)."""
    t = golden("builders")["domino/aztec2/min"]
    for model in ("domino", "domino_cftp"):
        ends = [po.walk_fast(model, t, 60, key).tobytes() for key in range(1600)]
        assert _uniform_pvalue(ends, 8) > P_MIN


def test_fast_lozenge_chains_are_uniform_on_hex2():
    """The 2 x 2 x 2 hexagon has 20 lozenge tilings (MacMahon)."""
    t = golden("builders")["lozenge/hex2_0/min"]
    ends = [po.walk_fast("lozenge", t, 90, 1000 + key).tobytes() for key in range(2000)]
    assert _uniform_pvalue(ends, 20) > P_MIN


def test_fast_cftp_samples_are_uniform_on_aztec2():
    b = golden("builders")
    tmax, tmin = b["domino/aztec2/max"], b["domino/aztec2/min"]
    out = []
    for seed in range(800):
        t, trials, total, ok = po.cftp(tmax, tmin, 8, seed, fast=True)
        assert ok
        out.append(t.tobytes())
    assert _uniform_pvalue(out, 8) > P_MIN


def test_fast_mode_depends_on_key_and_chain_only_through_the_counter():
    t = golden("builders")["lozenge/hex10_2/min"]
    a = po.walk_fast("lozenge", t, 300, 7)
    assert np.array_equal(a, po.walk_fast("lozenge", t, 300, 7))
    assert not np.array_equal(a, po.walk_fast("lozenge", t, 300, 8))
    assert not np.array_equal(a, po.walk_fast("lozenge", t, 300, 7, chain=1))
    assert not np.array_equal(a, po.walk_fast("lozenge", t, 300, 7 + (1 << 32)))


def test_fast_epochs_compose():
    """An epoch walk equals walking the epochs one after the other."""
    t = golden("builders")["domino/aztec8/min"]
    two = po.walk_fast("domino_cftp", t, [40, 25], [5, 9])
    one = po.walk_fast("domino_cftp", po.walk_fast("domino_cftp", t, 40, 5), 25, 9)
    assert np.array_equal(two, one)
