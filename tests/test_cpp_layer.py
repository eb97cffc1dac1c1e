"""The header-only C++ layer with the reference's names (Tilers.hpp) compiles
against include/ and links librt_b200.so; its builders agree with the
reference (CPU), its walks with the oracle (GPU)."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden
from oracle import pyoracle as po


def _build(tmp_path) -> str:
    from randomtilings_b200 import _capi

    lib = _capi.library_path()
    _capi.load()
    exe = str(tmp_path / "tilers_example")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "tilers_example.cpp"), "-o", exe, lib,
                    f"-Wl,-rpath,{os.path.dirname(lib)}"], check=True)
    return exe


def _read(path) -> dict:
    out = {}
    for line in open(path):
        parts = line.split()
        out[parts[0]] = np.array(parts[2:], dtype=np.int64)
    return out


def test_cpp_layer_builders(tmp_path):
    exe = _build(tmp_path)
    out = str(tmp_path / "b.txt")
    svg = str(tmp_path / "t.svg")
    subprocess.run([exe, "builders", out, svg], check=True)
    got, b = _read(out), golden("builders")
    assert np.array_equal(got["cone"], b["tridimer/cone10_3/tiling"])
    assert os.path.getsize(svg) > 1000
    assert np.array_equal(got["lozenge_max"], b["lozenge/hex10_2/max"])
    assert np.array_equal(got["lozenge_hmax"], b["lozenge/hex10_2/hmax"])
    d = b["domino/aztec13/domain"]
    assert got["aztec_min"].size == (2 * 12 + 6) ** 2 and d.size == (2 * 13 + 5) ** 2
    lo, hi = po.sixv_dwbc(6)
    assert np.array_equal(got["sixv_max"], hi)
    assert np.array_equal(got["sixv_asm_max"].reshape(6, 6), np.fliplr(np.eye(6, dtype=np.int64)))


@pytest.mark.gpu
def test_cpp_layer_walks(tmp_path):
    exe = _build(tmp_path)
    out = str(tmp_path / "w.txt")
    subprocess.run([exe, "walk", out], check=True)
    got, b = _read(out), golden("builders")
    assert np.array_equal(got["lozenge_walk"], po.lozenge_walk(b["lozenge/hex10_2/max"], 1000, 42))
    lw = (np.array([[1.0, 0.4], [1.6, 0.8]]), np.array([[0.5, 1.2], [2.0, 1.0]]), np.array([[1.5, 0.7], [0.9, 1.1]]))
    assert np.array_equal(got["lozenge_weighted"], po.lozenge_walk_weighted(b["lozenge/hex10_2/max"], [1000], [42], *lw))
    assert np.array_equal(got["cone_walk"], po.tridimer_walk(b["tridimer/cone10_3/tiling"], 800, 9))
    assert np.array_equal(got["aztec_epochs"],
                          po.domino_walk_epochs(got["aztec_min"], [256, 128], [2718281, 345903], cftp=True))
    assert np.array_equal(got["sixv_walk"], po.sixv_walk(po.sixv_dwbc(20)[0], 300, 5))
    assert np.array_equal(got["sixv_cftp"], po.sixv_cftp(8, 8, 3)[0])
    wh, wv = np.array([[1.0, 0.3], [0.5, 2.0]]), np.array([[0.7, 1.5], [1.0, 0.2]])
    assert np.array_equal(got["aztec_weighted"],
                          po.domino_walk_weighted(got["aztec_min"], [256, 128], [2718281, 345903], wh, wv))
