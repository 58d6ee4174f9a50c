"""The reference's API behaviour (tests/test_sparsesolv.py) on the B200 path,
with synthetic systems in place of NGSolve meshes."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def poisson():
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(10)
    b = P.random_rhs(A.shape[0], 0)
    fd = P.boundary_freedofs_7pt(10)
    return A, b, fd


def test_properties(poisson):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd)
    assert s.method == "ICCG"
    assert abs(s.tol - 1e-10) < 1e-15
    assert s.maxiter == 1000
    assert abs(s.shift - 1.05) < 1e-10
    assert s.save_best_result is True
    assert s.save_residual_history is False
    assert s.auto_shift is False
    assert s.diagonal_scaling is False
    assert s.divergence_check is False
    assert abs(s.divergence_threshold - 1000.0) < 1e-10
    assert s.divergence_count == 100
    assert s.use_abmc is False and s.abmc_block_size == 4 and s.abmc_num_colors == 4
    s.method = "SGSMRTR"
    assert s.method == "SGSMRTR"
    s.tol = 1e-8
    assert abs(s.tol - 1e-8) < 1e-15
    s.maxiter = 500
    assert s.maxiter == 500
    s.auto_shift = True
    assert s.auto_shift is True
    s.diagonal_scaling = True
    assert s.diagonal_scaling is True
    s.divergence_check = True
    assert s.divergence_check is True
    s.divergence_threshold = 10.0
    assert abs(s.divergence_threshold - 10.0) < 1e-10
    s.divergence_count = 5
    assert s.divergence_count == 5


def test_invalid_method(poisson):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    s = ss.SparseSolvSolver(A, method="INVALID", freedofs=fd)
    with pytest.raises(RuntimeError, match="Unknown method 'INVALID'"):
        s.Solve(b, np.zeros_like(b))


def test_operator_interface(poisson):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, tol=1e-10, maxiter=2000)
    x1 = s * b
    x2 = np.zeros_like(b)
    s.Solve(b, x2)
    assert np.linalg.norm(x1 - x2) / max(np.linalg.norm(x1), 1e-30) < 1e-6


def test_residual_history(poisson):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, save_residual_history=True)
    r = s.Solve(b, np.zeros_like(b))
    assert r.converged and len(r.residual_history) > 0
    assert r.residual_history[-1] < r.residual_history[0]
    s2 = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, save_residual_history=False)
    assert len(s2.Solve(b, np.zeros_like(b)).residual_history) == 0


def test_save_best_result(poisson):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, save_best_result=True, save_residual_history=True)
    r = s.Solve(b, np.zeros_like(b))
    assert r.converged and r.final_residual <= r.residual_history[0]


def test_divergence_check_early_termination():
    """A singular (pure Neumann) Laplacian with an inconsistent RHS stagnates;
    the stagnation check stops CG long before maxiter."""
    import scipy.sparse as sp
    import sparsesolv_ngsolve as ss
    n = 200
    main = np.full(n, 2.0)
    main[0] = main[-1] = 1.0
    A = sp.diags([main, -np.ones(n - 1), -np.ones(n - 1)], [0, -1, 1], format="csr")
    b = np.ones(n)
    s = ss.SparseSolvSolver(A, method="CG", tol=1e-12, maxiter=5000)
    s.divergence_check = True
    s.divergence_threshold = 10.0
    s.divergence_count = 20
    r = s.Solve(b, np.zeros(n))
    assert r.iterations < 5000 and not r.converged


def test_typed_classes(poisson):
    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import problems as P
    A, b, fd = poisson
    assert type(ss.SparseSolvSolver(A)).__name__ == "SparseSolvSolverD"
    assert type(ss.ICPreconditioner(A)).__name__ == "ICPreconditionerD"
    Ac = P.complex_shifted(A, 1j)
    assert type(ss.SparseSolvSolver(Ac)).__name__ == "SparseSolvSolverC"
    assert type(ss.ICPreconditioner(Ac)).__name__ == "ICPreconditionerC"
    assert type(ss.COCRSolver(Ac, None)).__name__ == "COCRSolverC"
    assert type(ss.COCRSolver(A, None)).__name__ == "COCRSolverD"


def test_abmc_vs_level_schedule(poisson):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    xs = []
    for abmc in (False, True):
        s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, tol=1e-12, use_abmc=abmc)
        x = np.zeros_like(b)
        assert s.Solve(b, x).converged
        xs.append(x)
    assert np.linalg.norm(xs[0] - xs[1]) / np.linalg.norm(xs[0]) < 1e-6


@pytest.mark.parametrize("bs", [2, 4, 8, 16])
def test_abmc_block_sizes(poisson, bs):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, use_abmc=True, abmc_block_size=bs)
    assert s.Solve(b, np.zeros_like(b)).converged


def test_abmc_path_switch(poisson):
    """ICPreconditioner: switching use_abmc takes effect at the next Update()."""
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    A, b, fd = poisson
    p = ss.ICPreconditioner(A, freedofs=fd)
    y0 = p * b
    p.use_abmc = True
    p.Update()
    y1 = p * b
    p.use_abmc = False
    p.Update()
    y2 = p * b
    ref_l, _ = O.ic_mult(A, b, O.default_config(), freedofs=fd)
    ref_a, _ = O.ic_mult(A, b, O.default_config(use_abmc=1), freedofs=fd)
    assert np.abs(y0 - ref_l).max() < 1e-12 * np.abs(ref_l).max()
    assert np.abs(y1 - ref_a).max() < 1e-12 * np.abs(ref_a).max()
    assert np.array_equal(y0, y2)


def test_auto_shift_reported(poisson):
    import sparsesolv_ngsolve as ss
    from oracle import oracle as O
    A, b, fd = poisson
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, shift=0.3)
    s.auto_shift = True
    s._cfg.min_diagonal_threshold = 2.0
    r = s.Solve(b, np.zeros_like(b))
    cfg = O.default_config(shift_parameter=0.3, auto_shift=1, min_diagonal_threshold=2.0)
    _, sh = O.ic_mult(A, b, cfg, freedofs=fd)
    assert r.converged
    assert abs(r.actual_shift - sh) < 1e-12 and r.actual_shift > 0.3


def test_missing_diagonal_raises():
    import scipy.sparse as sp
    import sparsesolv_ngsolve as ss
    A = sp.csr_matrix(np.array([[0.0, 1.0], [1.0, 2.0]]))
    A.eliminate_zeros()
    s = ss.SparseSolvSolver(A, method="ICCG")
    with pytest.raises(RuntimeError, match="missing diagonal"):
        s.Solve(np.ones(2), np.zeros(2))


def test_matrix_modified_in_place_is_reread(poisson):
    import sparsesolv_ngsolve as ss
    A, b, fd = poisson
    A = A.copy()
    s = ss.SparseSolvSolver(A, method="ICCG")
    x1 = s * b
    A.data *= 2.0
    x2 = s * b
    assert np.linalg.norm(x1 - 2 * x2) / np.linalg.norm(x1) < 1e-8


@pytest.mark.gpu
def test_dev_calls_refuse_host_pointers():
    # the check runs before any kernel: a host pointer returns an error, no launch
    import ctypes

    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import _capi
    from sparsesolv_ngsolve import problems as P
    A = P.laplacian_7pt(6)
    m = ss._Matrix(A)
    x = np.ones(A.shape[0])
    y = np.zeros(A.shape[0])
    lib = _capi.load()
    with pytest.raises(ValueError, match="host memory"):
        _capi.check(lib.ssv_matrix_spmv_dev(m.h, _capi.vptr(x), _capi.vptr(y)))
    res = _capi.ssv_result()
    cfg = _capi.default_config()
    fd = np.ones(A.shape[0], np.uint8)
    with pytest.raises(ValueError, match="host memory"):
        _capi.check(lib.ssv_pcg_solve_dev(m.h, None, _capi.u8ptr(fd), ctypes.byref(cfg), _capi.vptr(x),
                                          _capi.vptr(y), ctypes.byref(res), None, 0))
