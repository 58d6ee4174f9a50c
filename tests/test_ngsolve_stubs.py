"""The NGSolve-shaped inputs of the Python layer, with stand-ins that have
NGSolve's method names (NGSolve itself is not installed): a SparseMatrix
read through `CSR()` (values, column indices, row pointers) with `height` /
`width`, a BitArray of FreeDofs read through `len()` and `[]`, and a
BaseVector read and written through `FV().NumPy()`. CPU tests check the
adapters against the scipy / numpy forms; the GPU tests run whole solves
with the stand-ins and require the results of the same solves with scipy and
numpy inputs, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

import sparsesolv_ngsolve as ss
from sparsesolv_ngsolve import hcurl as H
from sparsesolv_ngsolve import problems as P


class StubSparseMatrix:
    """NGSolve SparseMatrix<double> / <Complex>: CSR() -> (vals, cols, rows)."""

    def __init__(self, A):
        A = sp.csr_matrix(A)
        A.sort_indices()
        self._A = A
        self.height, self.width = A.shape

    def CSR(self):
        return memoryview(self._A.data), memoryview(self._A.indices), memoryview(self._A.indptr)


class StubBitArray:
    def __init__(self, mask):
        self._m = [bool(v) for v in mask]

    def __len__(self):
        return len(self._m)

    def __getitem__(self, i):
        return self._m[i]


class _FV:
    def __init__(self, a):
        self._a = a

    def NumPy(self):
        return self._a


class StubBaseVector:
    def __init__(self, a):
        self.data = np.array(a)

    def FV(self):
        return _FV(self.data)


def test_csr_adapter_matches_scipy():
    A = P.laplacian_7pt(6)
    ip, ix, data, cplx, shape = ss._csr_arrays(StubSparseMatrix(A))
    B = sp.csr_matrix(A)
    assert not cplx and shape == B.shape
    assert np.array_equal(ip, B.indptr) and np.array_equal(ix, B.indices) and np.array_equal(data, B.data)
    Ac = (A + 1j * sp.eye(A.shape[0])).tocsr()
    ip, ix, data, cplx, shape = ss._csr_arrays(StubSparseMatrix(Ac))
    assert cplx and data.dtype == np.complex128
    assert np.array_equal(data, sp.csr_matrix(Ac).data)


def test_freedofs_and_vector_adapters():
    mask = np.array([1, 0, 1, 1, 0], dtype=bool)
    assert np.array_equal(ss._freedofs_array(StubBitArray(mask), 5), mask.astype(np.uint8))
    with pytest.raises(ValueError):
        ss._freedofs_array(StubBitArray(mask), 6)
    v = StubBaseVector(np.zeros(5))
    view = ss._vec_view(v)
    view[...] = 3.0
    assert np.all(v.data == 3.0)


@pytest.mark.gpu
def test_iccg_with_ngsolve_shaped_inputs():
    A = P.laplacian_7pt(12)
    b = P.random_rhs(A.shape[0], 3)
    fd = np.ones(A.shape[0], dtype=bool)
    fd[::17] = False
    s1 = ss.SparseSolvSolver(A, method="ICCG", tol=1e-10, maxiter=500, freedofs=fd)
    x1 = np.zeros_like(b)
    r1 = s1.Solve(b, x1)
    s2 = ss.SparseSolvSolver(StubSparseMatrix(A), method="ICCG", tol=1e-10, maxiter=500, freedofs=StubBitArray(fd))
    xv = StubBaseVector(np.zeros_like(b))
    r2 = s2.Solve(StubBaseVector(b), xv)
    assert r1.converged and r2.converged and r1.iterations == r2.iterations
    assert np.array_equal(x1, xv.data)


@pytest.mark.gpu
def test_complex_ams_cocr_with_ngsolve_shaped_inputs():
    d = H.eddy_current(6, nu_r_core=1.0, mass_eps=1.0, sigma=1e5, freq=1e3)
    fd = d["freedofs"].astype(bool)

    def run(wrap):
        mat = StubSparseMatrix if wrap else (lambda M: M)
        fds = StubBitArray(fd) if wrap else fd
        pre = ss.ComplexCompactAMSPreconditioner(mat(d["a_real"]), mat(d["G"]), freedofs=fds, coord_x=d["coords"][0],
                                                 coord_y=d["coords"][1], coord_z=d["coords"][2])
        inv = ss.COCRSolver(mat(d["A"]), pre, freedofs=fds, maxiter=500, tol=1e-10)
        if wrap:
            x = StubBaseVector(np.zeros(d["A"].shape[0], dtype=np.complex128))
            inv.Mult(StubBaseVector(d["f"]), x)
            return inv.iterations, x.data
        x = np.zeros(d["A"].shape[0], dtype=np.complex128)
        inv.Mult(d["f"], x)
        return inv.iterations, x

    it1, x1 = run(False)
    it2, x2 = run(True)
    assert it1 == it2 and np.array_equal(x1, x2)
