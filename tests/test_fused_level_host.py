"""The fused V-cycle level products (R = P^T (I - A D^-1) for the down sweep,
U = [D^-1 (2I - A D^-1) | (I - D^-1 A) P] for the up sweep) are built on the
host; this CPU test compiles the host set-up source with a small test driver
(tests/host/fused_level_check.cpp) and compares both products with the
step-by-step level (first sweep, residual, restriction; prolongation, post
sweep) on random sparse levels, to 1e-13."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ngsolve-sparsesolv_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_fused_level_matches_step_by_step():
    out = os.path.join(ROOT, "tests", "host", "_build")
    os.makedirs(out, exist_ok=True)
    exe = os.path.join(out, "fused_level_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, os.path.join(ROOT, "tests", "host", "fused_level_check.cpp"),
                    os.path.join(CSRC, "amg_setup.cpp"), "-lpthread", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("shapes ok") == 6, r.stdout
