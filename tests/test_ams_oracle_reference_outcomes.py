"""The AMS restatement (oracle/ams_oracle.cpp) against the reference's own AMS
test outcomes, the only pins its tests hold for this part
(tests/test_sparsesolv.py:1228-1259, 1312-1343), on synthetic Kuhn-mesh
systems of the same kind: CompactAMS + CG on curl-curl + 0.01 mass (tol 1e-8,
maxiter 200) within 1e-4 of a direct solve, and ComplexCompactAMS (auxiliary
curl-curl + 1.0 mass) + COCR on curl-curl + 1j mass (tol 1e-6) in fewer than
500 iterations (and within 1e-4 of a direct solve). The GPU counterpart is
tests/test_gpu_ams_reference_outcomes.py."""
from __future__ import annotations

import numpy as np
import scipy.sparse.linalg as spla

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H


def _system():
    m = H.kuhn_mesh(8)
    Ke, Me = H.element_matrices(m)
    ones = np.ones(m.tets.shape[0])
    K, M = H.assemble(m, ones, Ke), H.assemble(m, ones, Me)
    fd = H.boundary_freedofs(m)
    f = H.loop_source(m, z_levels=(0.5,), squares=((0.15, 0.85), (0.2, 0.8))) * fd
    return K, M, fd, f, H.gradient_matrix(m), (m.coords[:, 0].copy(), m.coords[:, 1].copy(), m.coords[:, 2].copy())


def _direct(A, fd, b):
    free = np.flatnonzero(fd.astype(bool))
    x = np.zeros(A.shape[0], dtype=np.result_type(A.dtype, b.dtype))
    x[free] = spla.spsolve(A.tocsr()[free][:, free].tocsc(), b[free])
    return x


def test_oracle_reproduces_reference_ams_outcomes():
    K, M, fd, f, G, c = _system()
    A = (K + 0.01 * M).tocsr()
    x, r, _ = O.AmsOracle(A, G, fd, *c).pcg(f, config=O.default_config(tolerance=1e-8, max_iterations=200))
    xd = _direct(A, fd, f)
    assert r.converged and np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-4
    Ac = (K.astype(np.complex128) + 1j * M.astype(np.complex128)).tocsr()
    xc, it, _ = O.AmsOracle((K + M).tocsr(), G, fd, *c).cocr(Ac, f.astype(np.complex128), freedofs=fd, maxiter=500,
                                                             tol=1e-6)
    xcd = _direct(Ac, fd, f.astype(np.complex128))
    assert np.linalg.norm(xc) > 0 and it < 500
    assert np.linalg.norm(xc - xcd) / np.linalg.norm(xcd) < 1e-4
