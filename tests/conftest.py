"""Shared test set-up: import paths, the `gpu` marker, golden fixtures."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "ngsolve-sparsesolv_b200"))

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_small.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN, allow_pickle=False)


def golden_system(g, name):
    import scipy.sparse as sp
    ip = g[f"sys/{name}/indptr"]
    ix = g[f"sys/{name}/indices"]
    data = g[f"sys/{name}/data"]
    n = ip.shape[0] - 1
    A = sp.csr_matrix((data, ix, ip), shape=(n, n))
    b = g[f"sys/{name}/b"]
    fd = g[f"sys/{name}/fd"] if f"sys/{name}/fd" in g.files else None
    return A, b, fd


def golden_cases(g):
    names = sorted({k.split("/")[1] for k in g.files if k.startswith("case/")})
    out = []
    for c in names:
        info = g[f"case/{c}/info"]
        out.append((c, str(info[0]), str(info[1]), eval(str(info[2]))))  # noqa: S307 (own fixture)
    return out
