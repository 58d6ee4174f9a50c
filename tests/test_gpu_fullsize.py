"""Full-size parity of the benchmark configurations against the restatement
(AMS oracle + the reference's CG / COCRSolverNGS semantics), on the systems
the bench measures:

* config 2: real magnetostatic curl-curl on the 40^3 Kuhn mesh (462,520
  edges), Compact AMS + CG, FP64 and the FP32-preconditioner form;
* config 3: complex eddy current on the 64^3 Kuhn mesh (1,872,064 edges),
  ComplexCompactAMS + COCR to 1e-10, FP64 and the mixed form (fp32_nodal
  preconditioner under refined COCR);
* config 4: one column of the 40^3 eddy-current family (8 frequencies x 4
  sources), the single FP64 solve and the batched mixed form.

Each test prints the measured iteration counts, true residuals and solution
errors. Bars: iterations within 2% of the oracle's (FP64 forms), the true
residual at or below the tolerance where the stopping rule is the true
residual (CG's recurrence residual tracks it; refined COCR stops on it), and
the solution error within the bound each docstring gives. These systems are
ill-conditioned (iron nu_r 1e-3 next to air, mass weight 1e-6: cond
1e8..1e11), so rounding-order differences of 1e-16 between the device's
reductions and the host's sequential sums reach the solution at about
cond x 1e-16, and a residual-level stop at 1e-10 leaves a forward error of up
to cond x 1e-10. Where that forward error exceeds a fixed bar (the complex
64^3 and 40^3 eddy-current systems: GPU and oracle solutions differ by
~2e-6 while both stop at the same iteration with the same true residual),
the bar is relative to the oracle's own accuracy: against a solution refined
to a true residual of 1e-12 (refined FP64 COCR, its residual checked here
on the host), the GPU's solution must be at least as accurate as the
oracle's, within a factor 2."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import oracle as O
from sparsesolv_ngsolve import hcurl as H

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _threads():
    O.AmsOracle.set_threads(os.cpu_count() or 1)


def _rel(x, xo):
    return float(np.linalg.norm(x - xo) / np.linalg.norm(xo))


def _true_res(A, fd, x, b):
    fdm = fd.astype(bool)
    return float(np.linalg.norm((b - A @ np.where(fdm, x, 0))[fdm]) / np.linalg.norm(b[fdm]))


def test_config2_ams_cg_40():
    """FP64 form: iterations within 2%, solution within 1e-6 relative (2-norm)
    of the oracle's; FP32 form: iterations within 2 of the FP64 oracle's,
    solution within 1e-6; both true residuals <= 1.05 tol."""
    import sparsesolv_ngsolve as ss
    d = H.magnetostatic(40)
    _threads()
    o = O.AmsOracle(d["A"], d["G"], d["freedofs"], *d["coords"])
    xo, ro, _ = o.pcg(d["f"], config=O.default_config(tolerance=TOL, max_iterations=500))
    assert ro.converged
    pre = ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                      coord_y=d["coords"][1], coord_z=d["coords"][2])
    out = {}
    for prec in ("fp64", "fp32"):
        pre.precision = prec
        inv = ss.PCGSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=500, tol=TOL)
        x = np.zeros(d["A"].shape[0])
        r = inv.Solve(d["f"], x)
        out[prec] = (r.iterations, _true_res(d["A"], d["freedofs"], x, d["f"]), _rel(x, xo))
        assert r.converged
    tro = _true_res(d["A"], d["freedofs"], xo, d["f"])
    print(f"config 2 (40^3 AMS+CG): oracle {ro.iterations} it, true res {tro:.3e}; "
          + "; ".join(f"{k} {v[0]} it, true res {v[1]:.3e}, error {v[2]:.2e}" for k, v in out.items()))
    it64, tr64, e64 = out["fp64"]
    assert abs(it64 - ro.iterations) <= max(1, int(0.02 * ro.iterations))
    assert tr64 <= 1.05 * TOL and e64 <= 1e-6
    it32, tr32, e32 = out["fp32"]
    assert abs(it32 - ro.iterations) <= 2
    assert tr32 <= 1.05 * TOL and e32 <= 1e-6


def _accurate(ss, A, pre, fd, b):
    """A solution to a true relative residual <= 1e-12 (refined FP64 COCR on
    the FP64 preconditioner), checked on the host."""
    inv = ss.MixedCOCRSolver(A, pre, freedofs=fd, maxiter=6000, tol=1e-12, restart_drop=1e-5)
    x = inv * b
    assert inv.converged and _true_res(A, fd, x, b) <= 1.05e-12
    return x


def test_config3_eddy_cocr_64():
    """Plain FP64 COCR: iterations within 2% of the oracle's, true residual
    within 2x of the oracle's (both stop on the recurrence residual or the
    absolute breakdown test), error against the 1e-12 solution at most 2x the
    oracle's (and within 1e-5 of the oracle's solution). Mixed form: true
    residual <= tol, error against the 1e-12 solution at most 2x the oracle's."""
    import sparsesolv_ngsolve as ss
    d = H.eddy_current(64)
    _threads()
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    xo, ito, _ = o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=3000, tol=TOL)
    del o
    tro = _true_res(d["A"], d["freedofs"], xo, d["f"])
    pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.COCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=3000, tol=TOL)
    x = inv * d["f"]
    tr = _true_res(d["A"], d["freedofs"], x, d["f"])
    e = _rel(x, xo)
    xa = _accurate(ss, d["A"], pre, d["freedofs"], d["f"])
    ea, eoa = _rel(x, xa), _rel(xo, xa)
    pre.precision = "fp32_nodal"
    invm = ss.MixedCOCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=3000, tol=TOL, restart_drop=1e-5)
    xm = invm * d["f"]
    trm = _true_res(d["A"], d["freedofs"], xm, d["f"])
    em, ema = _rel(xm, xo), _rel(xm, xa)
    print(f"config 3 (64^3 eddy, COCR): oracle {ito} it, true res {tro:.3e}, error vs 1e-12 solution {eoa:.2e}; "
          f"GPU FP64 {inv.iterations} it, true res {tr:.3e}, error vs oracle {e:.2e}, vs 1e-12 solution {ea:.2e}; "
          f"mixed {invm.iterations} it / {invm.cycles} cycles, true res {trm:.3e}, error vs oracle {em:.2e}, "
          f"vs 1e-12 solution {ema:.2e}")
    assert abs(inv.iterations - ito) <= max(1, int(0.02 * ito))
    assert tr <= max(2 * tro, TOL) and e <= 1e-5 and ea <= 2 * eoa
    assert invm.converged and trm <= TOL and ema <= 2 * eoa


def test_config4_family_column_40():
    """One column (f = 3, source 0) of the 40^3 family: the single FP64 COCR
    within 2% of the oracle's iterations, its error against the 1e-12 solution
    at most 2x the oracle's (and within 1e-5 of the oracle's solution); the
    batched mixed solve of the whole family brings that column (and every
    other) to a true residual <= tol, its error against the 1e-12 solution at
    most 2x the oracle's."""
    import sparsesolv_ngsolve as ss
    d = H.eddy_family(40, nrhs=4)
    f, r = 3, 0
    _threads()
    o = O.AmsOracle(d["a_real"][f], d["G"], d["freedofs"], *d["coords"])
    xo, ito, _ = o.cocr(d["A"][f], d["B"][f, r], freedofs=d["freedofs"], maxiter=1000, tol=TOL)
    pres = [ss.ComplexCompactAMSPreconditioner(a, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                               coord_y=d["coords"][1], coord_z=d["coords"][2])
            for a in d["a_real"]]
    inv = ss.COCRSolver(d["A"][f], pres[f], freedofs=d["freedofs"], maxiter=1000, tol=TOL)
    x = inv * d["B"][f, r]
    e = _rel(x, xo)
    xa = _accurate(ss, d["A"][f], pres[f], d["freedofs"], d["B"][f, r])
    ea, eoa = _rel(x, xa), _rel(xo, xa)
    for p in pres:
        p.precision = "fp32_nodal"
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=1500,
                              tol=TOL, restart_drop=1e-5)
    X = bs.Solve(d["B"])
    em, ema = _rel(X[f, r], xo), _rel(X[f, r], xa)
    trs = [_true_res(d["A"][g], d["freedofs"], X[g, q], d["B"][g, q]) for g in range(8) for q in range(4)]
    print(f"config 4 (40^3 family, column f={f} r={r}): oracle {ito} it, error vs 1e-12 solution {eoa:.2e}; "
          f"GPU FP64 {inv.iterations} it, error vs oracle {e:.2e}, vs 1e-12 solution {ea:.2e}; batched mixed "
          f"{int(bs.iterations[f, r])} it, error vs oracle {em:.2e}, vs 1e-12 solution {ema:.2e}, max true res "
          f"over 32 columns {max(trs):.3e}, cycles {bs.last_timing['cycles']}")
    assert abs(inv.iterations - ito) <= max(1, int(0.02 * ito)) and e <= 1e-5 and ea <= 2 * eoa
    assert bs.converged.all() and max(trs) <= TOL and ema <= 2 * eoa
