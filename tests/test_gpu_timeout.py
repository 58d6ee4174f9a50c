"""The watchdog of the device-looped solves: every iterative solve loops its
iteration graph on the device, and the loop control stops it after a bounded
number of loop bodies (maxiter + 4 by default) with SSV_ERR_TIMEOUT, so a
state that never reports done cannot keep the GPU busy. Here the cap is set
far below the iterations a solve needs (ssv_set_loop_guard), which makes the
guard fire in every solver family; the solve returns the error, nothing
hangs, and the next solve on the same context (cap restored) succeeds."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from sparsesolv_ngsolve import hcurl as H
from sparsesolv_ngsolve import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture()
def guard():
    from sparsesolv_ngsolve import _capi
    lib = _capi.load()
    lib.ssv_set_loop_guard(3)
    yield lib
    lib.ssv_set_loop_guard(0)


def _after(fn):
    """fn() with the default cap must work again on the same context."""
    from sparsesolv_ngsolve import _capi
    _capi.load().ssv_set_loop_guard(0)
    return fn()


@pytest.mark.parametrize("method", ["ICCG", "CG", "COCR", "SGSMRTR"])
def test_sparsesolv_solver_guard_fires(guard, method):
    import sparsesolv_ngsolve as ss
    A = P.laplacian_7pt(10)
    b = P.random_rhs(A.shape[0], 0)
    s = ss.SparseSolvSolver(A, method=method, tol=1e-12, maxiter=200)
    with pytest.raises(RuntimeError, match="loop guard"):
        s.Solve(b, np.zeros_like(b))
    r = _after(lambda: s.Solve(b, np.zeros_like(b)))
    assert r.iterations > 3


def test_cocr_and_refined_cocr_guard_fire(guard):
    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import _capi
    d = H.eddy_current(6)
    pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2])
    m = ss._Matrix(d["A"])
    b = np.ascontiguousarray(d["f"])
    x = np.zeros_like(b)
    it = ctypes.c_int32()
    fd = np.ascontiguousarray(d["freedofs"].astype(np.uint8))
    rc = guard.ssv_cocr_solve(m.h, pre._h, _capi.u8ptr(fd), 200, 1e-10, 0, _capi.vptr(b), _capi.vptr(x),
                              ctypes.byref(it))
    assert rc == _capi.SSV_ERR_TIMEOUT and b"loop guard" in guard.ssv_last_error()
    inv = ss.MixedCOCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=200, tol=1e-10)
    with pytest.raises(RuntimeError, match="loop guard"):
        inv * d["f"]
    _after(lambda: inv * d["f"])
    assert inv.converged and inv.iterations > 3


def test_pcg_guard_fires(guard):
    import sparsesolv_ngsolve as ss
    d = H.magnetostatic(6, nu_iron=1.0, mass_eps=1.0)
    pre = ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                      coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.PCGSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=200, tol=1e-10)
    with pytest.raises(RuntimeError, match="loop guard"):
        inv.Solve(d["f"], np.zeros(d["A"].shape[0]))
    r = _after(lambda: inv.Solve(d["f"], np.zeros(d["A"].shape[0])))
    assert r.converged


def test_batched_guard_fires(guard):
    import sparsesolv_ngsolve as ss
    d = H.eddy_family(6, freqs=[1e3, 1e4], nrhs=4, nu_r_core=1.0, mass_eps=1.0, sigma=1e5)
    pres = [ss.ComplexCompactAMSPreconditioner(a, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                               coord_y=d["coords"][1], coord_z=d["coords"][2])
            for a in d["a_real"]]
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=300,
                              tol=1e-10)
    with pytest.raises(RuntimeError, match="loop guard"):
        bs.Solve(d["B"])
    _after(lambda: bs.Solve(d["B"]))
    assert bs.converged.all()
