"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
from __future__ import annotations

import os
import re

from conftest import ROOT


def declared_functions() -> set[str]:
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(rt_[a-z0-9_]+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported():
    from randomtilings_b200 import _capi

    lib = _capi.load()
    missing = sorted(n for n in declared_functions() if not hasattr(lib, n))
    assert not missing, missing
    assert len(declared_functions()) > 20


def test_bindings_cover_the_headers():
    from randomtilings_b200 import _capi

    assert declared_functions() <= set(_capi.SIGNATURES), sorted(declared_functions() - set(_capi.SIGNATURES))


def test_version_without_gpu():
    from randomtilings_b200 import _capi

    assert b"sm_100a" in _capi.load().rt_version()
