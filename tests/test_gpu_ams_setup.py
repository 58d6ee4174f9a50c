"""The AMS / AMG set-up of Update() on the device against the restatement:
every level matrix A_l and interpolation P_l of the four subspace
hierarchies equals the oracle's bit for bit (same pattern, same values), on
the SI and well-conditioned magnetostatic and eddy-current systems, after
creation and after Update() with new values. The device set-up runs every
sum in the order of the host set-up (amg_setup.cpp), which the oracle's
restatement of compact_amg.hpp shares, with no fused multiply-adds."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu


def _same(M, Mo):
    return (M.shape == Mo.shape and np.array_equal(M.indptr, Mo.indptr) and np.array_equal(M.indices, Mo.indices)
            and np.array_equal(M.data, Mo.data))


def _check(p, o):
    for s in range(4):
        lv = p.levels(s)
        assert lv == o.levels(s), s
        for l in range(len(lv)):
            A = p.level_matrix(s, l, 0)
            assert p.on_device
            assert _same(A, o.level_matrix(s, l, 0)), (s, l, "A")
            if l + 1 < len(lv):
                assert _same(p.level_matrix(s, l, 1), o.level_matrix(s, l, 1)), (s, l, "P")


@pytest.mark.parametrize("case", ["mag_si", "mag_well", "eddy_si"])
def test_device_hierarchy_equals_oracle_bitwise(case):
    import sparsesolv_ngsolve as ss
    if case == "mag_si":
        d, key = H.magnetostatic(10), "A"
    elif case == "mag_well":
        d, key = H.magnetostatic(8, nu_iron=1.0, mass_eps=1.0), "A"
    else:
        d, key = H.eddy_current(8), "a_real"
    A = d[key]
    p = (ss.ComplexCompactAMSPreconditioner if key == "a_real" else ss.CompactAMSPreconditioner)(
        A, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0], coord_y=d["coords"][1], coord_z=d["coords"][2])
    o = O.AmsOracle(A, d["G"], d["freedofs"], *d["coords"])
    _check(p, o)
    # Update() with new values on the same pattern (the Newton-step use)
    B = A.copy()
    B.data = B.data * (1.0 + 0.25 * np.cos(np.arange(B.nnz)) ** 2)
    B = ((B + B.T) * 0.5).tocsr()
    B.sort_indices()
    B.indptr = B.indptr.astype(np.int32)
    B.indices = B.indices.astype(np.int32)
    p.Update(B)
    o2 = O.AmsOracle(B, d["G"], d["freedofs"], *d["coords"])
    _check(p, o2)


def test_device_setup_times_reported():
    import sparsesolv_ngsolve as ss
    d = H.magnetostatic(8)
    p = ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                    coord_y=d["coords"][1], coord_z=d["coords"][2])
    t = p.setup_times
    assert t["total"] > 0 and t["host_hierarchy"] > 0 and t["total"] >= t["host_hierarchy"]
    p.Update()
    t2 = p.setup_times
    print(f"set-up {t}, Update {t2}")
    assert t2["total"] > 0
