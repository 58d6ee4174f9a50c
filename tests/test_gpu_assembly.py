"""On-device assembly of the Kuhn-mesh HCurl matrices (ssv_hcurl_assemble,
hcurl.assemble_on_device) against the host assembly of the fixtures
(hcurl.assemble, hcurl.gradient_matrix): the same CSR patterns, G equal, K and
M equal up to the rounding of the element formulas (1e-12 of each matrix's
largest entry; both sum every entry in element order), with element-wise
coefficients (iron and copper regions of the eddy-current configuration)."""
from __future__ import annotations

import time

import numpy as np
import pytest

from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu


def _check(A, B, tol):
    A, B = A.tocsr(), B.tocsr()
    A.sort_indices()
    B.sort_indices()
    assert A.shape == B.shape
    assert np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices)
    err = np.abs(A.data - B.data).max() / np.abs(B.data).max()
    assert err <= tol, err
    return err


@pytest.mark.parametrize("nc", [3, 6, 10])
def test_device_assembly_matches_host(nc):
    m = H.kuhn_mesh(nc)
    Ke, Me = H.element_matrices(m)
    nu, sig = H._eddy_fields(m, 5.8e7, 1e-3)
    t0 = time.perf_counter()
    K, M, G = H.assemble_on_device(m, nu, sig)
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    Kh, Mh = H.assemble(m, nu, Ke), H.assemble(m, sig, Me)
    t_host = time.perf_counter() - t0
    ek = _check(K, Kh, 1e-12)
    em = _check(M, Mh, 1e-12)
    Gh = H.gradient_matrix(m)
    _check(G, Gh, 0.0)
    print(f"{nc}^3: K error {ek:.1e}, M error {em:.1e}; device {t_dev:.3f} s, host {t_host:.3f} s")


def test_device_assembly_unit_coefficients_and_symmetry():
    m = H.kuhn_mesh(5)
    Ke, Me = H.element_matrices(m)
    K, M, G = H.assemble_on_device(m)
    ones = np.ones(m.tets.shape[0])
    _check(K, H.assemble(m, ones, Ke), 1e-12)
    _check(M, H.assemble(m, ones, Me), 1e-12)
    assert abs(K - K.T).max() <= 1e-12 * abs(K).max()
    # curl grad = 0: K G = 0 to rounding
    assert abs(K @ G).max() <= 1e-10 * abs(K).max()
