"""Synthetic linear systems with the shapes of the solve path's workloads.

NGSolve is not required: these generators stand in for its assembly
(``BilinearForm.Assemble`` and ``SparseMatrix.CreateFromCOO``), producing
scipy CSR matrices with sorted column indices and summed duplicates, the
layout NGSolve hands to the reference (ngsolve/sparsesolv_precond.hpp:43-58).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def csr_from_coo(rows, cols, vals, n, m=None):
    """COO -> CSR with duplicates summed and columns sorted (CreateFromCOO)."""
    m = n if m is None else m
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, m)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    A.indptr = A.indptr.astype(np.int32)
    A.indices = A.indices.astype(np.int32)
    return A


def laplacian_7pt(nx: int, ny: int | None = None, nz: int | None = None,
                  dtype=np.float64):
    """7-point Laplacian on the interior nodes of an (nx+1)^3 grid.

    Diagonal 6, neighbours -1, homogeneous Dirichlet outside. For nx = 64
    this is 262,144 unknowns and 1,810,432 nonzeros.
    """
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64).reshape(nz, ny, nx)
    rows = [idx.ravel()]
    cols = [idx.ravel()]
    vals = [np.full(n, 6.0)]
    for axis in range(3):
        for sh in (-1, 1):
            a = idx
            src = np.moveaxis(a, 2 - axis, 0)
            if sh == -1:
                r, c = src[1:], src[:-1]
            else:
                r, c = src[:-1], src[1:]
            rows.append(r.ravel())
            cols.append(c.ravel())
            vals.append(np.full(r.size, -1.0))
    A = csr_from_coo(np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), n)
    return A.astype(dtype)


def laplacian_5pt(nx: int, ny: int | None = None, dtype=np.float64):
    """5-point Laplacian on an nx-by-ny interior grid (diag 4, off -1)."""
    ny = nx if ny is None else ny
    n = nx * ny
    idx = np.arange(n, dtype=np.int64).reshape(ny, nx)
    rows = [idx.ravel()]
    cols = [idx.ravel()]
    vals = [np.full(n, 4.0)]
    for r, c in ((idx[:, 1:], idx[:, :-1]), (idx[:, :-1], idx[:, 1:]),
                 (idx[1:, :], idx[:-1, :]), (idx[:-1, :], idx[1:, :])):
        rows.append(r.ravel())
        cols.append(c.ravel())
        vals.append(np.full(r.size, -1.0))
    A = csr_from_coo(np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), n)
    return A.astype(dtype)


def random_rhs(n: int, seed: int = 0, dtype=np.float64):
    """uniform[-1,1] right-hand side from numpy.random.default_rng(seed)."""
    rng = np.random.default_rng(seed)
    if np.dtype(dtype).kind == "c":
        return (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex128)
    return rng.uniform(-1.0, 1.0, n)


def complex_shifted(A, shift: complex):
    """Complex-symmetric A + shift*I (a mass-like complex term)."""
    n = A.shape[0]
    B = (A.astype(np.complex128) + shift * sp.identity(n, dtype=np.complex128, format="csr")).tocsr()
    B.sort_indices()
    B.indptr = B.indptr.astype(np.int32)
    B.indices = B.indices.astype(np.int32)
    return B


def boundary_freedofs_7pt(nx: int):
    """Free-DOF mask marking the outermost layer of an nx^3 grid constrained."""
    f = np.ones((nx, nx, nx), dtype=np.uint8)
    f[0, :, :] = f[-1, :, :] = 0
    f[:, 0, :] = f[:, -1, :] = 0
    f[:, :, 0] = f[:, :, -1] = 0
    return f.ravel()
