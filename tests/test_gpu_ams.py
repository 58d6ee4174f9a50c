"""Compact AMS / ComplexCompactAMS on the GPU against the AMS oracle: same AMG
hierarchies, same preconditioner application, same CG / COCR iteration counts
(tests/test_sparsesolv.py:1228-1373 behaviour on synthetic Kuhn-mesh systems).

Tolerances. Two kinds of systems are used. The well-conditioned ones
(nu contrast 1, mass weight 1: cond(A) ~ 3e3) carry the parity bar itself:
applies to 1e-11, iteration counts within 2%, solutions to 1e-8 relative.
The SI systems of the benchmarks (iron nu_r = 1e-3, mass weight 1e-6) have
cond(A) ~ 1e8..1e11: a 1e-16 rounding difference between the device's
reduction order and the sequential host sums grows to ~1e-8 of max|y| in an
apply (measured), so applies are compared at 1e-7 there; the Krylov solves
must still match the oracle's iteration counts within 2% and reach the same
true residual. COCR on the SI eddy-current system is what exposed a coarse
solve done through an explicit pseudo-inverse (it stalls at a true residual
of 1e-2): the coarsest levels are solved through the kept LDL^T factors."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[6, 10])
def mag(request):
    return H.magnetostatic(request.param)


@pytest.fixture(scope="module")
def eddy():
    return H.eddy_current(8)


APPLY_RTOL_ILL = 1e-7     # SI systems, cond ~ 1e8 and above (see module docstring)
APPLY_RTOL_WELL = 1e-11   # cond ~ 3e3


@pytest.fixture(scope="module")
def mag_well():
    return H.magnetostatic(8, nu_iron=1.0, mass_eps=1.0)


@pytest.fixture(scope="module")
def eddy_well():
    return H.eddy_current(8, nu_r_core=1.0, mass_eps=1.0, sigma=1e5, freq=1e3)


def _ams(d, complex_form=False, **kw):
    import sparsesolv_ngsolve as ss
    if complex_form:
        return ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"],
                                                  coord_x=d["coords"][0], coord_y=d["coords"][1],
                                                  coord_z=d["coords"][2], **kw)
    return ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                       coord_y=d["coords"][1], coord_z=d["coords"][2], **kw)


def test_hierarchy_matches_oracle(mag):
    p = _ams(mag)
    o = O.AmsOracle(mag["A"], mag["G"], mag["freedofs"], *mag["coords"])
    for s in range(4):
        assert p.levels(s) == o.levels(s), s


@pytest.mark.parametrize("cycle_type", [1, 7])
def test_apply_matches_oracle(mag, cycle_type):
    p = _ams(mag, cycle_type=cycle_type)
    o = O.AmsOracle(mag["A"], mag["G"], mag["freedofs"], *mag["coords"], cycle_type=cycle_type)
    rng = np.random.default_rng(3)
    for _ in range(2):
        b = rng.standard_normal(mag["A"].shape[0])
        y = p * b
        yo = o.apply(b)
        assert np.abs(y - yo).max() <= APPLY_RTOL_ILL * np.abs(yo).max()


@pytest.mark.parametrize("cycle_type", [1, 7])
def test_apply_matches_oracle_well_conditioned(mag_well, cycle_type):
    d = mag_well
    p = _ams(d, cycle_type=cycle_type)
    o = O.AmsOracle(d["A"], d["G"], d["freedofs"], *d["coords"], cycle_type=cycle_type)
    b = np.random.default_rng(5).standard_normal(d["A"].shape[0])
    yo = o.apply(b)
    assert np.abs(p * b - yo).max() <= APPLY_RTOL_WELL * np.abs(yo).max()


def test_complex_apply_matches_oracle(eddy):
    p = _ams(eddy, complex_form=True)
    o = O.AmsOracle(eddy["a_real"], eddy["G"], eddy["freedofs"], *eddy["coords"])
    rng = np.random.default_rng(4)
    f = rng.standard_normal(eddy["A"].shape[0]) + 1j * rng.standard_normal(eddy["A"].shape[0])
    u = p * f
    uo = o.apply_complex(f)
    assert np.abs(u - uo).max() <= APPLY_RTOL_ILL * np.abs(uo).max()


def test_complex_apply_ragged_hierarchies():
    """At 18^3 (1 kHz, nu_r = 0.1 in the core, mass weight 1) the z nodal
    hierarchy has one level fewer than the x and y ones; the three nodal
    V-cycles still run in one launch chain, each hierarchy skipping the levels
    it does not have. This system is ragged yet insensitive to rounding (a
    1e-15 input perturbation moves the oracle's apply by 2e-13), so the apply
    is held to the well-conditioned bar."""
    d = H.eddy_current(18, freq=1e3, nu_r_core=0.1, mass_eps=1.0)
    p = _ams(d, complex_form=True)
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    counts = [len(o.levels(s)) for s in range(1, 4)]
    assert len(set(counts)) > 1, counts
    assert [len(p.levels(s)) for s in range(4)] == [len(o.levels(s)) for s in range(4)]
    rng = np.random.default_rng(7)
    f = rng.standard_normal(d["A"].shape[0]) + 1j * rng.standard_normal(d["A"].shape[0])
    uo = o.apply_complex(f)
    assert np.abs(p * f - uo).max() <= APPLY_RTOL_WELL * np.abs(uo).max()


def test_complex_apply_well_conditioned(eddy_well):
    d = eddy_well
    p = _ams(d, complex_form=True)
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    rng = np.random.default_rng(6)
    f = rng.standard_normal(d["A"].shape[0]) + 1j * rng.standard_normal(d["A"].shape[0])
    uo = o.apply_complex(f)
    assert np.abs(p * f - uo).max() <= APPLY_RTOL_WELL * np.abs(uo).max()


def test_ams_cg_parity_well_conditioned(mag_well):
    import sparsesolv_ngsolve as ss
    d = mag_well
    inv = ss.PCGSolver(d["A"], _ams(d), freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    x = np.zeros(d["A"].shape[0])
    r = inv.Solve(d["f"], x)
    o = O.AmsOracle(d["A"], d["G"], d["freedofs"], *d["coords"])
    xo, ro, _ = o.pcg(d["f"], config=O.default_config(tolerance=1e-10, max_iterations=500))
    assert r.converged and ro.converged
    assert abs(r.iterations - ro.iterations) <= max(1, int(0.02 * ro.iterations))
    assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()


def test_complex_cocr_parity_well_conditioned(eddy_well):
    import sparsesolv_ngsolve as ss
    d = eddy_well
    inv = ss.COCRSolver(d["A"], _ams(d, complex_form=True), freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    x = inv * d["f"]
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    xo, it, _ = o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    assert abs(inv.iterations - it) <= max(1, int(0.02 * it))
    assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()


def test_ams_cg_matches_oracle(mag):
    import sparsesolv_ngsolve as ss
    p = _ams(mag)
    inv = ss.PCGSolver(mag["A"], p, freedofs=mag["freedofs"], maxiter=500, tol=1e-10, save_residual_history=True)
    x = np.zeros(mag["A"].shape[0])
    r = inv.Solve(mag["f"], x)
    o = O.AmsOracle(mag["A"], mag["G"], mag["freedofs"], *mag["coords"])
    xo, ro, ho = o.pcg(mag["f"], config=O.default_config(tolerance=1e-10, max_iterations=500,
                                                          save_residual_history=1))
    assert r.converged and ro.converged
    assert abs(r.iterations - ro.iterations) <= max(1, int(0.02 * ro.iterations))
    assert np.abs(x - xo).max() <= 1e-6 * np.abs(xo).max()
    fd = mag["freedofs"].astype(bool)
    res = (mag["f"] - mag["A"] @ np.where(fd, x, 0))[fd]
    assert np.linalg.norm(res) / np.linalg.norm(mag["f"]) <= 1e-10 * 1.01


def test_complex_ams_cocr_matches_oracle(eddy):
    import sparsesolv_ngsolve as ss
    p = _ams(eddy, complex_form=True)
    inv = ss.COCRSolver(eddy["A"], p, freedofs=eddy["freedofs"], maxiter=500, tol=1e-8)
    x = inv * eddy["f"]
    o = O.AmsOracle(eddy["a_real"], eddy["G"], eddy["freedofs"], *eddy["coords"])
    xo, it, _ = o.cocr(eddy["A"], eddy["f"], freedofs=eddy["freedofs"], maxiter=500, tol=1e-8)
    fd = eddy["freedofs"].astype(bool)
    res = (eddy["f"] - eddy["A"] @ np.where(fd, x, 0))[fd]
    reso = (eddy["f"] - eddy["A"] @ np.where(fd, xo, 0))[fd]
    nf = np.linalg.norm(eddy["f"][fd])
    assert np.linalg.norm(res) / nf <= max(1e-8, 2 * np.linalg.norm(reso) / nf)
    assert abs(inv.iterations - it) <= max(1, int(0.02 * it))
    Ar = eddy["a_real"]
    e = np.where(fd, x - xo, 0)
    x0 = np.where(fd, xo, 0)
    assert np.sqrt(abs(np.vdot(e, Ar @ e))) <= 1e-4 * np.sqrt(abs(np.vdot(x0, Ar @ x0)))


def test_update_same_values_reproduces(mag):
    import sparsesolv_ngsolve as ss
    p = _ams(mag)
    inv = ss.PCGSolver(mag["A"], p, freedofs=mag["freedofs"], maxiter=500, tol=1e-10)
    x1 = inv * mag["f"]
    it1 = inv.iterations
    p.Update()
    x2 = inv * mag["f"]
    assert abs(inv.iterations - it1) <= 1
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x1) < 1e-6


def test_update_new_matrix_and_dimension_check(mag):
    import scipy.sparse as sp
    p = _ams(mag)
    A2 = mag["A"].copy()
    A2.data *= 3.0
    p.Update(A2)
    o = O.AmsOracle(A2, mag["G"], mag["freedofs"], *mag["coords"])
    b = np.random.default_rng(0).standard_normal(A2.shape[0])
    yo = o.apply(b)
    assert np.abs(p * b - yo).max() <= APPLY_RTOL_ILL * np.abs(yo).max()
    with pytest.raises(ValueError, match="does not match original"):
        p.Update(sp.identity(5, format="csr"))


def test_coordinate_mismatch_raises(mag):
    with pytest.raises(RuntimeError, match="coordinate size mismatch"):
        import sparsesolv_ngsolve as ss
        ss.CompactAMSPreconditioner(mag["A"], mag["G"], freedofs=mag["freedofs"], coord_x=[0.0], coord_y=[0.0],
                                    coord_z=[0.0])


def test_typed_names_and_flag(mag, eddy):
    import sparsesolv_ngsolve as ss
    assert ss.has_compact_ams() is True
    assert type(_ams(mag)).__name__ == "CompactAMSPreconditionerImpl"
    assert type(_ams(eddy, complex_form=True)).__name__ == "ComplexCompactAMSPreconditionerImpl"


# ---------------------------------------------------------------------------
# FP32-preconditioner form (new): FP32 hierarchy and cycle, FP64 Krylov. The
# oracle is the FP64 path; each test states the error it allows against it.
# ---------------------------------------------------------------------------

def test_precision_switch_roundtrip(mag):
    p = _ams(mag)
    b = np.random.default_rng(7).standard_normal(mag["A"].shape[0])
    y64 = p * b
    p.precision = "fp32"
    assert p.precision == "fp32"
    y32 = p * b
    # the accuracy of the FP32 form is checked on the well-conditioned system
    # below: here the gradient space amplifies FP32 rounding by ~1e8
    assert np.all(np.isfinite(y32))
    p.precision = "fp64"
    assert p.precision == "fp64"
    # the re-upload re-runs the lanes autotuner, which may pick another
    # summation split: equal to rounding (amplified as in the SI applies)
    assert np.abs(p * b - y64).max() <= APPLY_RTOL_ILL * np.abs(y64).max()
    with pytest.raises(ValueError):
        p.precision = "fp16"


def test_fp32_apply_well_conditioned(mag_well):
    d = mag_well
    p = _ams(d, precision="fp32")
    o = O.AmsOracle(d["A"], d["G"], d["freedofs"], *d["coords"])
    b = np.random.default_rng(5).standard_normal(d["A"].shape[0])
    yo = o.apply(b)
    # FP32 storage and arithmetic through ~20 passes: 1e-4 relative (stated)
    assert np.linalg.norm(p * b - yo) <= 1e-4 * np.linalg.norm(yo)


def test_fp32_ams_cg_reaches_fp64_tolerance(mag):
    import sparsesolv_ngsolve as ss
    p64 = _ams(mag)
    p32 = _ams(mag, precision="fp32")
    fd = mag["freedofs"].astype(bool)
    xs, its = [], []
    for p in (p64, p32):
        inv = ss.PCGSolver(mag["A"], p, freedofs=mag["freedofs"], maxiter=500, tol=1e-10)
        x = np.zeros(mag["A"].shape[0])
        r = inv.Solve(mag["f"], x)
        assert r.converged
        res = (mag["f"] - mag["A"] @ np.where(fd, x, 0))[fd]
        assert np.linalg.norm(res) / np.linalg.norm(mag["f"]) <= 1e-10 * 1.01  # FP64 outer recurrence
        xs.append(x)
        its.append(r.iterations)
    assert its[1] <= 1.5 * its[0] + 2
    # solution error of the mixed form against the FP64 solution, in the
    # energy norm CG minimises (stated bound); the near-kernel gradient
    # components, which the 1e-6 mass term barely weights, are not bounded
    A = mag["A"]
    e = np.where(fd, xs[1] - xs[0], 0)
    x0 = np.where(fd, xs[0], 0)
    assert np.sqrt(e @ (A @ e)) <= 1e-6 * np.sqrt(x0 @ (A @ x0))


def test_fp32_complex_apply_well_conditioned(eddy_well):
    # FP32 hierarchies inside the complex cycle: close to the FP64 cycle (stated
    # bound). COCR itself is not run with this form: its preconditioned-residual
    # recurrence assumes an exactly linear preconditioner, and FP32 rounding
    # stops it near a true residual of 1e-7 (the FP64 oracle with only its output
    # rounded to FP32 behaves the same), so the batched and single COCR forms
    # use FP64 preconditioners.
    d = eddy_well
    p64 = _ams(d, complex_form=True)
    p32 = _ams(d, complex_form=True, precision="fp32")
    rng = np.random.default_rng(8)
    f = rng.standard_normal(d["A"].shape[0]) + 1j * rng.standard_normal(d["A"].shape[0])
    u64 = p64 * f
    assert np.linalg.norm(p32 * f - u64) <= 1e-5 * np.linalg.norm(u64)


@pytest.mark.parametrize("complex_form", [False, True])
def test_lockstep_nodal_cycles_and_branches_agree(mag_well, eddy_well, monkeypatch, complex_form):
    # by default the three nodal V-cycles run as one chain of launches over
    # all three hierarchies; SSV_AMS_TRI=0 runs them as three graph branches
    d = eddy_well if complex_form else mag_well
    rng = np.random.default_rng(12)
    n = d["A"].shape[0]
    b = rng.standard_normal(n) + (1j * rng.standard_normal(n) if complex_form else 0)
    monkeypatch.setenv("SSV_AMS_TRI", "0")
    y_br = _ams(d, complex_form=complex_form) * b
    monkeypatch.setenv("SSV_AMS_TRI", "1")
    y_tri = _ams(d, complex_form=complex_form) * b
    assert np.abs(y_tri - y_br).max() <= APPLY_RTOL_WELL * np.abs(y_br).max()
    o = O.AmsOracle(d["a_real"] if complex_form else d["A"], d["G"], d["freedofs"], *d["coords"])
    yo = o.apply_complex(b) if complex_form else o.apply(b)
    assert np.abs(y_tri - yo).max() <= APPLY_RTOL_WELL * np.abs(yo).max()
