"""The reference's own AMS test outcomes, on synthetic Kuhn-mesh systems of
the same kind (tests/test_sparsesolv.py there assembles them with NGSolve,
absent here):

* CompactAMS + CG on curl-curl + 0.01 mass, tol 1e-8, maxiter 200: the
  solution within 1e-4 relative of a direct solve (:1228-1259);
* ComplexCompactAMS (auxiliary curl-curl + 1.0 mass, ndof_complex given) +
  COCR on curl-curl + 1j mass, tol 1e-6: a nonzero solution in fewer than 500
  iterations (:1312-1343); checked here against a direct solve too;
* ComplexCompactAMS with ndof_complex = 0 derives it from the matrix and
  applies to complex vectors (:1345-1373)."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mesh():
    m = H.kuhn_mesh(8)
    Ke, Me = H.element_matrices(m)
    ones = np.ones(m.tets.shape[0])
    K = H.assemble(m, ones, Ke)
    M = H.assemble(m, ones, Me)
    fd = H.boundary_freedofs(m)
    f = H.loop_source(m, z_levels=(0.5,), squares=((0.15, 0.85), (0.2, 0.8))) * fd
    G = H.gradient_matrix(m)
    return dict(m=m, K=K, M=M, fd=fd, f=f, G=G,
                coords=(m.coords[:, 0].copy(), m.coords[:, 1].copy(), m.coords[:, 2].copy()))


def _direct(A, fd, f):
    free = np.flatnonzero(fd.astype(bool))
    Af = A.tocsr()[free][:, free].tocsc()
    x = np.zeros(A.shape[0], dtype=np.result_type(A.dtype, f.dtype))
    x[free] = spla.spsolve(Af, f[free])
    return x


def test_compact_ams_cg_against_direct_solve(mesh):
    import sparsesolv_ngsolve as ss
    d = mesh
    A = (d["K"] + 0.01 * d["M"]).tocsr()
    pre = ss.CompactAMSPreconditioner(A, d["G"], freedofs=d["fd"], coord_x=d["coords"][0],
                                      coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.PCGSolver(A, pre, freedofs=d["fd"], tol=1e-8, maxiter=200)
    x = np.zeros(A.shape[0])
    r = inv.Solve(d["f"], x)
    xd = _direct(A, d["fd"], d["f"])
    rel = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    print(f"CompactAMS+CG: {r.iterations} iterations, rel_err = {rel:.2e}")
    assert r.converged
    assert rel < 1e-4


def test_complex_compact_ams_cocr_converges(mesh):
    import sparsesolv_ngsolve as ss
    d = mesh
    A = (d["K"].astype(np.complex128) + 1j * d["M"].astype(np.complex128)).tocsr()
    a_real = (d["K"] + 1.0 * d["M"]).tocsr()
    pre = ss.ComplexCompactAMSPreconditioner(a_real, d["G"], freedofs=d["fd"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2],
                                             ndof_complex=A.shape[0])
    inv = ss.COCRSolver(A, pre, freedofs=d["fd"], maxiter=500, tol=1e-6)
    x = inv * d["f"].astype(np.complex128)
    xd = _direct(A, d["fd"], d["f"].astype(np.complex128))
    rel = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    print(f"ComplexCompactAMS+COCR: {inv.iterations} iterations, rel_err = {rel:.2e}")
    assert np.linalg.norm(x) > 0
    assert inv.iterations < 500
    assert rel < 1e-4


def test_complex_compact_ams_derives_ndof(mesh):
    import sparsesolv_ngsolve as ss
    d = mesh
    a_real = (d["K"] + 1.0 * d["M"]).tocsr()
    pre = ss.ComplexCompactAMSPreconditioner(a_real, d["G"], freedofs=d["fd"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2])
    n = a_real.shape[0]
    zero = np.zeros(n, dtype=np.complex128)
    out = np.full(n, 1.0 + 1.0j)
    pre.Mult(zero, out)
    assert np.array_equal(out, np.zeros(n, dtype=np.complex128))
    b = np.random.default_rng(4).standard_normal(n) + 1j * np.random.default_rng(5).standard_normal(n)
    y = pre * b
    assert y.dtype == np.complex128 and np.isfinite(y).all() and np.linalg.norm(y) > 0
