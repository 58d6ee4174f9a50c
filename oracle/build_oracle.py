"""Build recipe of the oracle (TEST INFRASTRUCTURE).

* ``oracle/_build/libssv_oracle.so``: the plain-C restatement (ssv_oracle.c).
* ``oracle/_ref/libssv_ref.so``: the reference's own headers
  (ksugahar/ngsolve-sparsesolv, include/sparsesolv, NGSolve-free half),
  driven by ref_driver.cpp. Built only where the reference checkout exists;
  the built file travels with the working tree to machines that lack it.

Run ``python oracle/build_oracle.py`` (``__graft_entry__.build()`` calls it).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_INCLUDE = os.environ.get("SSV_REFERENCE_INCLUDE", "/root/reference/include")
ORACLE_SO = os.path.join(HERE, "_build", "libssv_oracle.so")
AMS_SO = os.path.join(HERE, "_build", "libssv_ams_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libssv_ref.so")


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, "ssv_oracle.c"), os.path.join(HERE, "ssv_oracle_body.h"),
            os.path.join(HERE, "..", "include", "sparsesolv_b200.h")]
    if force or _stale(ORACLE_SO, srcs):
        os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
        _run(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-o", ORACLE_SO, srcs[0], "-lm"])
    return ORACLE_SO


def build_ams_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, "ams_oracle.cpp"), os.path.join(HERE, "..", "include", "sparsesolv_b200.h")]
    if force or _stale(AMS_SO, srcs):
        os.makedirs(os.path.dirname(AMS_SO), exist_ok=True)
        _run(["g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", AMS_SO, srcs[0]])
    return AMS_SO


def build_reference(force: bool = False) -> str | None:
    hdr = os.path.join(REF_INCLUDE, "sparsesolv", "sparsesolv.hpp")
    if not os.path.exists(hdr):
        return REF_SO if os.path.exists(REF_SO) else None
    src = os.path.join(HERE, "ref_driver.cpp")
    if force or _stale(REF_SO, [src]):
        os.makedirs(os.path.dirname(REF_SO), exist_ok=True)
        # -mavx2 -mfma as the reference's own CMakeLists.txt:98 uses (portable
        # to the GPU hosts; -march=native would not be)
        _run(["g++", "-std=c++17", "-O3", "-mavx2", "-mfma", "-fopenmp", "-fPIC", "-shared",
              "-I", REF_INCLUDE, "-o", REF_SO, src])
    return REF_SO


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_ams_oracle(force))
    print(build_reference(force))
