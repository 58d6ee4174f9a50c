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
GOLDEN_EDGE = os.path.join(ROOT, "tests", "golden", "golden_edge.npz")


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


def edge_cases():
    """The edge-input fixtures (tests/golden/gen_golden_edge.py): per case the
    matrix, b, the initial guess, the method, the config items and the
    reference's outputs."""
    import ast

    import scipy.sparse as sp
    g = np.load(GOLDEN_EDGE, allow_pickle=False)
    out = []
    for c in sorted({k.split("/")[0] for k in g.files}):
        ip, ix, data = g[f"{c}/indptr"], g[f"{c}/indices"], g[f"{c}/data"]
        n = ip.shape[0] - 1
        info = g[f"{c}/info"]
        conv, iters, fres = g[f"{c}/meta"]
        out.append(dict(case=c, A=sp.csr_matrix((data, ix, ip), shape=(n, n)), b=g[f"{c}/b"], x0=g[f"{c}/x0"],
                        method=str(info[0]), items=ast.literal_eval(str(info[1])), x=g[f"{c}/x"],
                        hist=g[f"{c}/hist"], converged=int(conv), iterations=int(iters), final_residual=fres))
    return out


def assert_same_outcome(case, converged, iterations, final_residual, x, hist):
    """The reference's outcome of an edge case: flags and counts equal, NaN
    where the reference has NaN, and elsewhere residuals to 1e-5 relative plus
    1e-9 of the initial residual (the bars of the main parity tests; with a
    zero b the normaliser is 1, so the last residuals are absolute rounding
    noise near 1e-14) and solutions to 1e-10 of their largest entry."""
    c = case["case"]
    assert int(converged) == case["converged"], c
    assert int(iterations) == case["iterations"], c
    hr = case["hist"]
    fin = ~np.isnan(hr)
    floor = 1e-9 * (abs(hr[fin][0]) if fin.any() else 1.0)
    fr = case["final_residual"]
    if np.isnan(fr):
        assert np.isnan(final_residual), (c, final_residual)
    elif fr > 1e300:
        assert final_residual == fr, (c, final_residual)
    else:
        assert abs(final_residual - fr) <= 1e-5 * fr + floor, (c, final_residual, fr)
    xr = case["x"]
    assert np.array_equal(np.isnan(x), np.isnan(xr)), c
    ok = ~np.isnan(xr)
    if ok.any():
        scale = max(np.abs(xr[ok]).max(), 1e-300)
        assert np.abs(x[ok] - xr[ok]).max() <= 1e-10 * scale + 1e-14, c
    assert len(hist) == len(hr), (c, len(hist), len(hr))
    h = np.asarray(hist, dtype=np.float64)
    assert np.array_equal(np.isnan(h), np.isnan(hr)), c
    np.testing.assert_allclose(h[fin], hr[fin], rtol=1e-5, atol=floor, err_msg=c)
