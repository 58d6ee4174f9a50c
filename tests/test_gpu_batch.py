"""Batched COCR over a frequency family (new form, no reference counterpart):
every column must reproduce the single-system COCRSolver with the same
ComplexCompactAMS preconditioner, whose own parity with the oracle is covered
in test_gpu_ams.py. On a well-conditioned family (nu contrast 1, mass weight
1) the bar is the parity bar: iterations within 2%, solutions to 1e-8
relative. The SI family is checked for convergence and the true residual."""
from __future__ import annotations

import numpy as np
import pytest

from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu

WELL = dict(nu_r_core=1.0, mass_eps=1.0, sigma=1e5)


@pytest.fixture(scope="module")
def fam_well():
    return H.eddy_family(6, freqs=[1e2, 1e3, 1e4], nrhs=4, **WELL)


def _pres(d, precision="fp64"):
    import sparsesolv_ngsolve as ss
    return [ss.ComplexCompactAMSPreconditioner(a, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                               coord_y=d["coords"][1], coord_z=d["coords"][2], precision=precision)
            for a in d["a_real"]]


def _single(d, pres, f, r, tol, maxiter=500):
    import sparsesolv_ngsolve as ss
    inv = ss.COCRSolver(d["A"][f], pres[f], freedofs=d["freedofs"], maxiter=maxiter, tol=tol)
    x = inv * d["B"][f, r]
    return x, inv.iterations


def _true_res(d, f, x, b):
    fd = d["freedofs"].astype(bool)
    res = (b - d["A"][f] @ np.where(fd, x, 0))[fd]
    return np.linalg.norm(res) / np.linalg.norm(b[fd])


def test_batch_matches_single_solves(fam_well):
    import sparsesolv_ngsolve as ss
    d = fam_well
    pres = _pres(d)
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=500,
                              tol=1e-10)
    X = bs.Solve(d["B"])
    assert X.shape == d["B"].shape
    assert bs.converged.all()
    for f in range(len(d["omegas"])):
        for r in range(4):
            xs, its = _single(d, pres, f, r, 1e-10)
            it = int(bs.iterations[f, r])
            assert abs(it - its) <= max(1, int(0.02 * its)), (f, r, it, its)
            assert np.abs(X[f, r] - xs).max() <= 1e-8 * np.abs(xs).max(), (f, r)
            assert _true_res(d, f, X[f, r], d["B"][f, r]) <= 1e-9


def test_batch_one_rhs_per_frequency(fam_well):
    import sparsesolv_ngsolve as ss
    d = fam_well
    pres = _pres(d)
    B1 = d["B"][:, :1].copy()
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=1, freedofs=d["freedofs"], tol=1e-10)
    X = bs.Solve(B1)
    for f in range(len(d["omegas"])):
        xs, its = _single(d, pres, f, 0, 1e-10)
        assert abs(int(bs.iterations[f, 0]) - its) <= max(1, int(0.02 * its))
        assert np.abs(X[f, 0] - xs).max() <= 1e-8 * np.abs(xs).max()


def test_batch_zero_column_and_constrained_dofs(fam_well):
    import sparsesolv_ngsolve as ss
    d = fam_well
    B = d["B"].copy()
    B[1, 2] = 0.0
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], _pres(d), nrhs=4, freedofs=d["freedofs"], tol=1e-10)
    X = bs.Solve(B)
    assert bs.iterations[1, 2] == 0 and not np.any(X[1, 2])
    fd = d["freedofs"].astype(bool)
    assert not np.any(X[:, :, ~fd])
    assert bs.converged.sum() == B.shape[0] * B.shape[1] - 1


def test_batch_residual_replacement(fam_well):
    import sparsesolv_ngsolve as ss
    d = fam_well
    pres = _pres(d)
    plain = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], tol=1e-10)
    plain.Solve(d["B"])
    rep = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], tol=1e-10,
                               residual_replacement=5)
    X = rep.Solve(d["B"])
    assert rep.converged.all()
    # with an exactly linear preconditioner the replaced value equals the recurrence's
    assert (np.abs(rep.iterations - plain.iterations) <= np.maximum(2, 0.1 * plain.iterations)).all()
    for f in range(len(d["omegas"])):
        for r in range(4):
            assert _true_res(d, f, X[f, r], d["B"][f, r]) <= 1e-9


def test_batch_without_preconditioner(fam_well):
    import sparsesolv_ngsolve as ss
    d = fam_well
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"][:1], [None], nrhs=4, freedofs=d["freedofs"], maxiter=60,
                              tol=1e-10)
    X = bs.Solve(d["B"][:1])
    inv = ss.COCRSolver(d["A"][0], None, freedofs=d["freedofs"], maxiter=60, tol=1e-10)
    x = inv * d["B"][0, 0]
    # 60 unpreconditioned steps, not converged: the two reduction orders drift apart slowly
    assert abs(int(bs.iterations[0, 0]) - inv.iterations) <= 1
    assert np.linalg.norm(X[0, 0] - x) <= 1e-4 * np.linalg.norm(x)


def test_batch_autotuner_record(fam_well):
    import sparsesolv_ngsolve as ss
    d = fam_well
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], _pres(d), nrhs=4, freedofs=d["freedofs"])
    t = bs.tuning
    assert len(t["candidates"]) >= 3 and {c[1] for c in t["candidates"]} == {4, 8, 16}
    assert t["chosen"] is not None
    assert t["chosen"][3] == min(c[3] for c in t["candidates"])
    F = len(d["omegas"])
    assert all(F % c[0] == 0 and c[0] * 4 <= 16 for c in t["candidates"])
    bs.Solve(d["B"])
    tm = bs.last_timing
    assert tm["device_ms"] > 0 and tm["loops"] >= bs.iterations.max() and tm["kernel_launches"] > 0


def test_batch_argument_errors(fam_well):
    import sparsesolv_ngsolve as ss
    d = fam_well
    pres = _pres(d)
    with pytest.raises(ValueError):
        ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=3, freedofs=d["freedofs"])
    with pytest.raises(ValueError):
        ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres[:2], nrhs=4, freedofs=d["freedofs"])
    real = ss.CompactAMSPreconditioner(d["a_real"][0], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                       coord_y=d["coords"][1], coord_z=d["coords"][2])
    with pytest.raises(TypeError):
        ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"][:1], [real], nrhs=4, freedofs=d["freedofs"])
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"])
    with pytest.raises(ValueError):
        bs.Solve(d["B"][:, :2])


def test_batch_si_family_converges():
    import sparsesolv_ngsolve as ss
    d = H.eddy_family(6, freqs=[1e3, 1e5], nrhs=4)
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], _pres(d), nrhs=4, freedofs=d["freedofs"], maxiter=800,
                              tol=1e-8)
    X = bs.Solve(d["B"])
    assert bs.converged.all()
    for f in range(2):
        for r in range(4):
            assert _true_res(d, f, X[f, r], d["B"][f, r]) <= 1e-6


def test_batch_columns_match_oracle(fam_well):
    """Every column of the plain batched solve against the restatement's
    COCRSolverNGS with the FP64 AMS oracle of its frequency: iterations within
    2%, solutions to 1e-8 relative (well-conditioned family)."""
    import sparsesolv_ngsolve as ss

    from oracle import oracle as O
    d = fam_well
    pres = _pres(d)
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=500,
                              tol=1e-10)
    X = bs.Solve(d["B"])
    for f in range(len(d["omegas"])):
        o = O.AmsOracle(d["a_real"][f], d["G"], d["freedofs"], *d["coords"])
        for r in range(4):
            xo, ito, _ = o.cocr(d["A"][f], d["B"][f, r], freedofs=d["freedofs"], maxiter=500, tol=1e-10)
            it = int(bs.iterations[f, r])
            assert abs(it - ito) <= max(1, int(0.02 * ito)), (f, r, it, ito)
            assert np.abs(X[f, r] - xo).max() <= 1e-8 * np.abs(xo).max(), (f, r)
