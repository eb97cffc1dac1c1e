"""The batched triangle-dimer kernel keeps the eight state arrays as bit
planes (csrc/rt_tdplane.cuh).  On the host, every bit-plane phase op must
give the integer rule's values (csrc/rt_tridimer.cuh) at every site of a
real chain: tests/cpp/tdplane_check.cpp compiles both for the host and
compares them phase by phase, starting from the state arrays the oracle
splits from a tiling."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden
from oracle import pyoracle as po


@pytest.fixture(scope="module")
def checker(tmp_path_factory) -> str:
    exe = str(tmp_path_factory.mktemp("tdplane") / "tdplane_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "randomtilings_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "tdplane_check.cpp"), "-o", exe], check=True)
    return exe


def _tilings():
    import randomtilings_b200 as rt

    yield "bibone hexagon 10", np.asarray(rt.TriangleDimerTiler.BiboneHexagon(10), dtype=np.int32)
    yield "ice-cream cone 10, 3", np.asarray(golden("builders")["tridimer/cone10_3/tiling"], dtype=np.int32)


@pytest.mark.parametrize("k", [0, 1])
def test_bit_plane_ops_equal_the_integer_rule(checker, tmp_path, k):
    name, t = list(_tilings())[k]
    arrays = po.tridimer_arrays(t)
    m = arrays.shape[1]
    path = str(tmp_path / "arrays.bin")
    np.ascontiguousarray(arrays, dtype=np.int32).tofile(path)
    out = subprocess.run([checker, path, str(m), "300"], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), (name, out.stdout, out.stderr)
    changed = int(out.stdout.split()[6])
    assert changed > 1000, (name, out.stdout)  # the chain moved: the comparison covered real flips


def test_bit_plane_ops_on_random_states(checker):
    """Every phase of the 30 moves on random states of each array's bit width:
    the digit sums' adder paths (conditions that overlap, which chains from
    valid tilings never produce) agree with the integer rule modulo the width
    the planes keep."""
    out = subprocess.run([checker, "random", "40", "3"], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), (out.stdout, out.stderr)


def test_oracle_split_fits_the_bit_planes():
    import randomtilings_b200 as rt

    a = po.tridimer_arrays(np.asarray(rt.TriangleDimerTiler.BiboneHexagon(12), dtype=np.int32))
    bits = [4, 4, 4, 6, 6, 9, 9, 9]
    for arr in range(8):
        assert a[arr].min() >= 0 and a[arr].max() < (1 << bits[arr]), arr
