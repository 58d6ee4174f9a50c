"""The set-up's host worker threads (csrc/host_threads.hpp) hand an exception
to the thread that joins them instead of ending the process: a small driver
compiled here with g++ checks run_threads (every job runs, the lowest failing
index's exception is rethrown after the join) and WorkerThread (join
rethrows, wait does not)."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ngsolve-sparsesolv_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_worker_exceptions_reach_the_caller():
    out = os.path.join(ROOT, "tests", "host", "_build")
    os.makedirs(out, exist_ok=True)
    exe = os.path.join(out, "threads_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC,
                    os.path.join(ROOT, "tests", "host", "threads_check.cpp"), "-o", exe], check=True, timeout=300)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
