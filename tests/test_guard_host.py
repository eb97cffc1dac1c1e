"""csrc/rt_guard.h, the wrapper every exported function runs its body
through: statuses pass unchanged, std::bad_alloc becomes RT_E_NOMEM and any
other exception RT_E_INVAL, so no C++ exception reaches a C caller.  Built
for the host and run.  No GPU."""
from __future__ import annotations

import os
import subprocess

from conftest import ROOT


def test_guard_maps_exceptions_to_statuses(tmp_path):
    exe = str(tmp_path / "guard_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "randomtilings_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "guard_check.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", (out.stdout, out.stderr)
