"""Compact AMS / ComplexCompactAMS on the GPU against the AMS oracle: same AMG
hierarchies, same preconditioner application, same CG / COCR iteration counts
(tests/test_sparsesolv.py:1228-1373 behaviour on synthetic Kuhn-mesh systems)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[6, 10])
def mag(request):
    return H.magnetostatic(request.param)


@pytest.fixture(scope="module")
def eddy():
    return H.eddy_current(8)


def _ams(d, complex_form=False, **kw):
    import sparsesolv_ngsolve as ss
    if complex_form:
        return ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"],
                                                  coord_x=d["coords"][0], coord_y=d["coords"][1],
                                                  coord_z=d["coords"][2], **kw)
    return ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                       coord_y=d["coords"][1], coord_z=d["coords"][2], **kw)


def test_hierarchy_matches_oracle(mag):
    p = _ams(mag)
    o = O.AmsOracle(mag["A"], mag["G"], mag["freedofs"], *mag["coords"])
    for s in range(4):
        assert p.levels(s) == o.levels(s), s


@pytest.mark.parametrize("cycle_type", [1, 7])
def test_apply_matches_oracle(mag, cycle_type):
    p = _ams(mag, cycle_type=cycle_type)
    o = O.AmsOracle(mag["A"], mag["G"], mag["freedofs"], *mag["coords"], cycle_type=cycle_type)
    rng = np.random.default_rng(3)
    for _ in range(2):
        b = rng.standard_normal(mag["A"].shape[0])
        y = p * b
        yo = o.apply(b)
        assert np.abs(y - yo).max() <= 1e-9 * np.abs(yo).max()


def test_complex_apply_matches_oracle(eddy):
    p = _ams(eddy, complex_form=True)
    o = O.AmsOracle(eddy["a_real"], eddy["G"], eddy["freedofs"], *eddy["coords"])
    rng = np.random.default_rng(4)
    f = rng.standard_normal(eddy["A"].shape[0]) + 1j * rng.standard_normal(eddy["A"].shape[0])
    u = p * f
    uo = o.apply_complex(f)
    assert np.abs(u - uo).max() <= 1e-9 * np.abs(uo).max()


def test_ams_cg_matches_oracle(mag):
    import sparsesolv_ngsolve as ss
    p = _ams(mag)
    inv = ss.PCGSolver(mag["A"], p, freedofs=mag["freedofs"], maxiter=500, tol=1e-10, save_residual_history=True)
    x = np.zeros(mag["A"].shape[0])
    r = inv.Solve(mag["f"], x)
    o = O.AmsOracle(mag["A"], mag["G"], mag["freedofs"], *mag["coords"])
    xo, ro, ho = o.pcg(mag["f"], config=O.default_config(tolerance=1e-10, max_iterations=500,
                                                          save_residual_history=1))
    assert r.converged and ro.converged
    assert abs(r.iterations - ro.iterations) <= max(1, int(0.02 * ro.iterations))
    assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()
    fd = mag["freedofs"].astype(bool)
    res = (mag["f"] - mag["A"] @ np.where(fd, x, 0))[fd]
    assert np.linalg.norm(res) / np.linalg.norm(mag["f"]) <= 1e-10 * 1.01


def test_complex_ams_cocr_matches_oracle(eddy):
    import sparsesolv_ngsolve as ss
    p = _ams(eddy, complex_form=True)
    inv = ss.COCRSolver(eddy["A"], p, freedofs=eddy["freedofs"], maxiter=500, tol=1e-8)
    x = inv * eddy["f"]
    o = O.AmsOracle(eddy["a_real"], eddy["G"], eddy["freedofs"], *eddy["coords"])
    xo, it, _ = o.cocr(eddy["A"], eddy["f"], freedofs=eddy["freedofs"], maxiter=500, tol=1e-8)
    assert abs(inv.iterations - it) <= max(1, int(0.02 * it))
    assert np.abs(x - xo).max() <= 1e-6 * np.abs(xo).max()


def test_update_same_values_reproduces(mag):
    import sparsesolv_ngsolve as ss
    p = _ams(mag)
    inv = ss.PCGSolver(mag["A"], p, freedofs=mag["freedofs"], maxiter=500, tol=1e-10)
    x1 = inv * mag["f"]
    it1 = inv.iterations
    p.Update()
    x2 = inv * mag["f"]
    assert abs(inv.iterations - it1) <= 1
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x1) < 1e-6


def test_update_new_matrix_and_dimension_check(mag):
    import scipy.sparse as sp
    p = _ams(mag)
    A2 = mag["A"].copy()
    A2.data *= 3.0
    p.Update(A2)
    o = O.AmsOracle(A2, mag["G"], mag["freedofs"], *mag["coords"])
    b = np.random.default_rng(0).standard_normal(A2.shape[0])
    assert np.abs(p * b - o.apply(b)).max() <= 1e-9 * np.abs(o.apply(b)).max()
    with pytest.raises(ValueError, match="does not match original"):
        p.Update(sp.identity(5, format="csr"))


def test_coordinate_mismatch_raises(mag):
    with pytest.raises(RuntimeError, match="coordinate size mismatch"):
        import sparsesolv_ngsolve as ss
        ss.CompactAMSPreconditioner(mag["A"], mag["G"], freedofs=mag["freedofs"], coord_x=[0.0], coord_y=[0.0],
                                    coord_z=[0.0])


def test_typed_names_and_flag(mag, eddy):
    import sparsesolv_ngsolve as ss
    assert ss.has_compact_ams() is True
    assert type(_ams(mag)).__name__ == "CompactAMSPreconditionerImpl"
    assert type(_ams(eddy, complex_form=True)).__name__ == "ComplexCompactAMSPreconditionerImpl"
