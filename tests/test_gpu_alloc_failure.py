"""Device-allocation failures, injected on the host: ssv_set_alloc_budget
refuses every allocation past a byte budget before CUDA is asked, so no GPU
memory is exhausted. A refused allocation ends the call with SSV_ERR_ALLOC,
raised as MemoryError (what the reference's pybind11 module makes of
std::bad_alloc), and the library stays usable: once the budget is lifted the
failed objects, or new ones, solve as a run that never failed does. Covered:
the AMS set-up with its worker threads at several budgets, a failed Update()
(the preconditioner then refuses to apply until an Update succeeds), the
first solve's work vectors, the ICCG set-up, and an Update() with a matrix of
another dimension (ValueError, nothing changed)."""
from __future__ import annotations

import numpy as np
import pytest

import sparsesolv_ngsolve as ss
from sparsesolv_ngsolve import _capi
from sparsesolv_ngsolve import hcurl as H
from sparsesolv_ngsolve import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture()
def budget():
    lib = _capi.load()

    def set_(b):
        lib.ssv_set_alloc_budget(int(b))

    yield set_
    lib.ssv_set_alloc_budget(-1)


@pytest.fixture(scope="module")
def mag():
    return H.magnetostatic(8, nu_iron=1.0, mass_eps=1.0)


def _ams(d):
    return ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                       coord_y=d["coords"][1], coord_z=d["coords"][2])


def _solve(d, pre):
    inv = ss.PCGSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    x = np.zeros(d["A"].shape[0])
    r = inv.Solve(d["f"], x)
    return int(r.iterations), x


@pytest.fixture(scope="module")
def baseline(mag):
    return _solve(mag, _ams(mag))


def _same(got, ref):
    its, x = got
    its0, x0 = ref
    assert abs(its - its0) <= 1, (its, its0)
    assert np.linalg.norm(x - x0) <= 1e-9 * np.linalg.norm(x0)


@pytest.mark.parametrize("nbytes", [0, 1 << 16, 1 << 20, 4 << 20, 16 << 20])
def test_ams_setup_refused_then_recovers(mag, baseline, budget, nbytes):
    budget(nbytes)
    failed = False
    try:
        pre = _ams(mag)
    except MemoryError as e:
        failed = True
        assert "allocation budget" in str(e)
    budget(-1)
    if not failed:  # the budget sufficed: the object must work as usual
        _same(_solve(mag, pre), baseline)
    _same(_solve(mag, _ams(mag)), baseline)
    if nbytes <= 1 << 20:
        assert failed


def test_failed_update_refuses_to_apply_until_an_update_succeeds(mag, baseline, budget):
    pre = _ams(mag)
    b = np.random.default_rng(0).standard_normal(mag["A"].shape[0])
    y0 = pre * b
    budget(0)
    with pytest.raises(MemoryError):
        pre.Update()
    budget(-1)
    with pytest.raises(RuntimeError):
        pre * b
    pre.Update()
    y1 = pre * b
    assert np.linalg.norm(y1 - y0) <= 1e-9 * np.linalg.norm(y0)
    _same(_solve(mag, pre), baseline)


def test_first_solve_work_vectors_refused_then_recover(mag, baseline, budget):
    pre = _ams(mag)
    inv = ss.PCGSolver(mag["A"], pre, freedofs=mag["freedofs"], maxiter=500, tol=1e-10)
    x = np.zeros(mag["A"].shape[0])
    budget(0)
    with pytest.raises(MemoryError):
        inv.Solve(mag["f"], x)
    budget(-1)
    x = np.zeros(mag["A"].shape[0])
    r = inv.Solve(mag["f"], x)
    _same((int(r.iterations), x), baseline)


def test_complex_cocr_refused_then_recovers(budget):
    d = H.eddy_current(6, nu_r_core=1.0, mass_eps=1.0, sigma=1e5, freq=1e3)

    def run():
        pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"],
                                                 coord_x=d["coords"][0], coord_y=d["coords"][1],
                                                 coord_z=d["coords"][2])
        inv = ss.COCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=1000, tol=1e-10)
        return inv, inv * d["f"]

    inv0, x0 = run()
    for nbytes in (0, 1 << 20):
        budget(nbytes)
        with pytest.raises(MemoryError):
            run()
        budget(-1)
    inv1, x1 = run()
    assert abs(inv1.iterations - inv0.iterations) <= 1
    assert np.linalg.norm(x1 - x0) <= 1e-9 * np.linalg.norm(x0)


def test_iccg_setup_refused_then_recovers(budget):
    A = P.laplacian_7pt(12)
    b = P.random_rhs(A.shape[0], seed=1)
    x0 = np.zeros(A.shape[0])
    solver = ss.SparseSolvSolver(A, method="ICCG", tol=1e-10, maxiter=1000)
    r0 = solver.Solve(b, x0)
    budget(0)
    with pytest.raises(MemoryError):
        ss.SparseSolvSolver(A, method="ICCG", tol=1e-10, maxiter=1000).Solve(b, np.zeros(A.shape[0]))
    budget(-1)
    x1 = np.zeros(A.shape[0])
    r1 = ss.SparseSolvSolver(A, method="ICCG", tol=1e-10, maxiter=1000).Solve(b, x1)
    assert r1.iterations == r0.iterations
    assert np.array_equal(x1, x0)


def test_update_with_other_dimension_raises_and_keeps_the_preconditioner(mag, baseline):
    pre = _ams(mag)
    other = H.magnetostatic(6, nu_iron=1.0, mass_eps=1.0)["A"]
    with pytest.raises(ValueError):
        pre.Update(other)
    _same(_solve(mag, pre), baseline)
