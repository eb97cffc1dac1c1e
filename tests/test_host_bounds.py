"""Sizes the host functions refuse: builder arguments whose arrays would pass
32,767 on a side (the side whose lozenge domain, 2 side^2 entries, still has
int32 indices) and array lengths that are negative, huge or not square.  Each
returns RT_E_INVAL without allocating anything.  No GPU."""
from __future__ import annotations

import ctypes

import pytest

from randomtilings_b200 import _capi

BIG = 2**31 - 1


def _call(name, *args):
    lib = _capi.load()
    n = ctypes.c_int64(-1)
    st = getattr(lib, name)(*args, None, 0, ctypes.byref(n))
    return st, n.value


@pytest.mark.parametrize("name,args", [
    ("rt_domino_rectangle", (BIG, 1)),
    ("rt_domino_rectangle", (32763, 1)),
    ("rt_domino_aztec", (BIG,)),
    ("rt_domino_aztec", (16382,)),
    ("rt_lozenge_almost_hex", (BIG, 0)),
    ("rt_lozenge_almost_hex", (16380, 0)),
    ("rt_lozenge_hexagon", (BIG, 1, 1)),
    ("rt_lozenge_hexagon", (1, BIG, BIG)),
    ("rt_lozenge_hexagon", (16380, 16380, 10)),
    ("rt_recttri_max_hex", (BIG,)),
    ("rt_recttri_min_hex", (16380,)),
    ("rt_tridimer_ice_cream_cone", (BIG, 0)),
    ("rt_tridimer_ice_cream_cone", (16380, 0)),
    ("rt_tridimer_hexagon", (BIG,)),
])
def test_builders_refuse_oversized_domains(name, args):
    st, n = _call(name, *args)
    assert st == _capi.RT_E_INVAL
    assert n == -1


@pytest.mark.parametrize("name,length", [
    ("rt_domino_domain_to_vertices", -4),
    ("rt_domino_domain_to_vertices", 2**63 - 1),
    ("rt_domino_domain_to_vertices", 32768**2),
    ("rt_lozenge_domain_to_vertices", 2 * 32768**2),
    ("rt_lozenge_domain_to_vertices", -8),
])
def test_array_lengths_out_of_range_are_refused(name, length):
    # a size query (out = NULL): nothing is read from the array
    dummy = (ctypes.c_int32 * 4)()
    st, n = _call(name, dummy, length)
    assert st == _capi.RT_E_INVAL
    assert n == -1


def test_largest_sizes_still_accepted_by_size_queries():
    dummy = (ctypes.c_int32 * 4)()
    st, n = _call("rt_domino_domain_to_vertices", dummy, 32767**2)
    assert st == _capi.RT_OK and n == 32768**2
