"""The Compact AMS oracle (C++ restatement of compact_amg.hpp / compact_ams.hpp /
complex_compact_ams.hpp) on synthetic Kuhn-mesh systems: the behaviour the
reference's own AMS tests pin (tests/test_sparsesolv.py:1228-1373), CPU only.
NGSolve is absent, so agreement with NGSolve itself is not checked here."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H


@pytest.fixture(scope="module")
def mag8():
    return H.magnetostatic(8)


def test_kuhn_sizes():
    m = H.kuhn_mesh(40)
    assert (m.nv, m.ne) == (68921, 462520)
    m = H.kuhn_mesh(3)
    assert np.isclose(m.vol.sum(), 1.0)


def test_whitney_exact_sequence(mag8):
    K = H.assemble(mag8["mesh"], np.ones(len(mag8["mesh"].vol)), mag8["Ke"])
    assert abs(K @ mag8["G"]).max() < 1e-12
    assert abs(mag8["G"].T @ mag8["f"]).max() < 1e-12


def test_ams_cg_converges(mag8):
    ams = O.AmsOracle(mag8["A"], mag8["G"], mag8["freedofs"], *mag8["coords"])
    x, res, hist = ams.pcg(mag8["f"], config=O.default_config(tolerance=1e-10, max_iterations=300,
                                                              save_residual_history=1))
    assert res.converged and res.iterations < 150
    fd = mag8["freedofs"].astype(bool)
    A = mag8["A"]
    r = (mag8["f"] - A @ np.where(fd, x, 0))[fd]
    assert np.linalg.norm(r) / np.linalg.norm(mag8["f"]) < 1e-9


def test_ams_preconditioner_symmetric_positive(mag8):
    ams = O.AmsOracle(mag8["A"], mag8["G"], mag8["freedofs"], *mag8["coords"])
    rng = np.random.default_rng(1)
    fd = mag8["freedofs"].astype(bool)
    u = rng.standard_normal(len(fd)) * fd
    v = rng.standard_normal(len(fd)) * fd
    Mu, Mv = ams.apply(u), ams.apply(v)
    assert abs(v @ Mu - u @ Mv) <= 1e-6 * abs(v @ Mu)
    assert u @ Mu > 0


def test_ams_update_reproduces(mag8):
    """Update() with the same values reproduces iterations (+-1) and solution (< 1e-6)."""
    ams = O.AmsOracle(mag8["A"], mag8["G"], mag8["freedofs"], *mag8["coords"])
    cfg = O.default_config(tolerance=1e-10, max_iterations=300)
    x1, r1, _ = ams.pcg(mag8["f"], config=cfg)
    ams.update(mag8["A"].data)
    x2, r2, _ = ams.pcg(mag8["f"], config=cfg)
    assert abs(r1.iterations - r2.iterations) <= 1
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x1) < 1e-6


def test_complex_ams_cocr_converges():
    e = H.eddy_current(8)
    ams = O.AmsOracle(e["a_real"], e["G"], e["freedofs"], *e["coords"])
    x, it, hist = ams.cocr(e["A"], e["f"], freedofs=e["freedofs"], maxiter=500, tol=1e-6)
    assert 0 < it < 500
    assert hist[-1] <= 1e-6
