"""Writes tests/golden/sixv.npz: regression vectors for the six-vertex model.

The reference names the model without code, so these vectors come from this
project's restatement (oracle/sixv_oracle.c), itself pinned by exact
enumeration (tests/test_sixv_oracle.py).  They hold the restatement's
results fixed, so that a later change to it shows as a failed CPU test
rather than as a GPU/oracle disagreement found only on a GPU:

* walk/<n>/<start>/<weights>: the heights after 40 sweeps (key 0x5EED + n,
  chain n mod 3) from the minimal or maximal domain-wall heights, uniform and
  weighted (a1..c2 = 1, 0.7, 1.6, 1.2, 2, 0.5), for n in 7, 24, 65;
* epochs/<n>: a walk of three epochs (5, 11, 2 sweeps; keys 3, 2**40 + 9,
  77) from the minimal heights;
* cftp/<n>/<seed>: the CFTP sample and its trial and sweep counts from
  first_sweeps 4.

Run from the repository root: python tests/golden/make_sixv_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

WEIGHTED = (1.0, 0.7, 1.6, 1.2, 2.0, 0.5)


def main() -> None:
    out = {}
    for n in (7, 24, 65):
        lo, hi = po.sixv_dwbc(n)
        for sname, start in (("min", lo), ("max", hi)):
            for wname, w in (("uniform", po.SIXV_UNIFORM), ("weighted", WEIGHTED)):
                out[f"walk/{n}/{sname}/{wname}"] = po.sixv_walk(start, 40, 0x5EED + n, chain=n % 3, w=w)
        out[f"epochs/{n}"] = po.sixv_walk(lo, [5, 11, 2], [3, 2**40 + 9, 77])
    for n, seed in ((6, 0), (10, 4), (16, 1)):
        h, trials, sweeps, ok = po.sixv_cftp(n, 4, seed)
        assert ok
        out[f"cftp/{n}/{seed}"] = h
        out[f"cftp/{n}/{seed}/counts"] = np.array([trials, sweeps], dtype=np.int64)
    path = os.path.join(ROOT, "tests", "golden", "sixv.npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in out.items()})
    print(f"wrote {path}: {len(out)} arrays")


if __name__ == "__main__":
    main()
