"""The COCR iteration's SpMV through the system matrix's sliced-ELL copy
(matrices of at least 65,536 rows; SSV_KRYLOV_SELL=0 keeps the CSR arrays).

The copy changes only the order in which each row's products are summed, so
against the CSR form (run in a child process with the switch off) the
iteration counts agree within one and the solutions within 1e-9 relative on
the well-conditioned 24^3 eddy-current system (cond ~ 3e3) and on the real
24^3 magnetostatic system with unit permeability; against the oracle the
counts agree within 2%. A change of the matrix values (the
Python layer re-reads them every solve) reaches the copy: the solution of
2A x = b is half that of A x = b."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-10
WELL = dict(nu_r_core=1.0, mass_eps=1.0, sigma=1e5, freq=1e3)

_CHILD = r"""
import json, os, sys
sys.path.insert(0, os.path.join(sys.argv[1], "ngsolve-sparsesolv_b200")); sys.path.insert(0, sys.argv[1])
import numpy as np
import sparsesolv_ngsolve as ss
from sparsesolv_ngsolve import hcurl as H
if sys.argv[3] == "complex":
    d = H.eddy_current(24, nu_r_core=1.0, mass_eps=1.0, sigma=1e5, freq=1e3)
    pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2])
else:
    d = H.magnetostatic(24, nu_iron=1.0, mass_eps=1.0)
    pre = ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                      coord_y=d["coords"][1], coord_z=d["coords"][2])
inv = ss.COCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=1000, tol=1e-10)
x = inv * d["f"]
np.save(sys.argv[2], x)
print(json.dumps({"iterations": inv.iterations}))
"""


@pytest.fixture(scope="module")
def well24():
    return H.eddy_current(24, **WELL)


def _solve(ss, d, A=None):
    pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.COCRSolver(d["A"] if A is None else A, pre, freedofs=d["freedofs"], maxiter=1000, tol=TOL)
    return inv, inv * d["f"]


def test_sell_matches_csr_form(well24, tmp_path):
    import sparsesolv_ngsolve as ss
    d = well24
    assert d["A"].shape[0] >= 65536
    inv, x = _solve(ss, d)
    out = tmp_path / "x_csr.npy"
    env = dict(os.environ, SSV_KRYLOV_SELL="0")
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, str(out), "complex"], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    it_csr = json.loads(r.stdout.strip().splitlines()[-1])["iterations"]
    x_csr = np.load(out)
    err = np.linalg.norm(x - x_csr) / np.linalg.norm(x_csr)
    print(f"sliced-ELL {inv.iterations} it, CSR {it_csr} it, difference {err:.2e}")
    assert abs(inv.iterations - it_csr) <= 1
    assert err <= 1e-9


def test_real_cocr_sell_matches_csr_form(tmp_path):
    """COCRSolver on a real system (the same kernel with real values)."""
    import sparsesolv_ngsolve as ss
    d = H.magnetostatic(24, nu_iron=1.0, mass_eps=1.0)
    assert d["A"].shape[0] >= 65536
    pre = ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                      coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.COCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=1000, tol=TOL)
    x = inv * d["f"]
    out = tmp_path / "x_csr_real.npy"
    env = dict(os.environ, SSV_KRYLOV_SELL="0")
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, str(out), "real"], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    it_csr = json.loads(r.stdout.strip().splitlines()[-1])["iterations"]
    x_csr = np.load(out)
    assert abs(inv.iterations - it_csr) <= 1
    assert np.linalg.norm(x - x_csr) <= 1e-9 * np.linalg.norm(x_csr)


def test_sell_iterations_match_oracle(well24):
    import sparsesolv_ngsolve as ss
    d = well24
    O.AmsOracle.set_threads(os.cpu_count() or 1)
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    xo, ito, _ = o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=1000, tol=TOL)
    inv, x = _solve(ss, d)
    err = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    print(f"GPU {inv.iterations} it, oracle {ito} it, error {err:.2e}")
    assert abs(inv.iterations - ito) <= max(1, int(0.02 * ito))
    assert err <= 1e-8


def test_value_change_reaches_copy(well24):
    import sparsesolv_ngsolve as ss
    d = well24
    A = d["A"].copy()
    pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.COCRSolver(A, pre, freedofs=d["freedofs"], maxiter=1000, tol=TOL)
    x1 = inv * d["f"]
    A.data *= 2.0  # in place: the solver re-reads the values
    x2 = inv * d["f"]
    assert np.linalg.norm(2.0 * x2 - x1) <= 1e-8 * np.linalg.norm(x1)
