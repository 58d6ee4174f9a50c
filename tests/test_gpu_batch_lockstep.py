"""With SSV_AMS_MULTI=1 the batched solver applies its per-frequency
ComplexCompactAMS cycles in lockstep (one launch chain for all frequencies'
V-cycles; a hierarchy with fewer levels skips the launches of the levels it
lacks); by default (SSV_AMS_MULTI=0) it applies them as parallel graph
branches. Both give the same columns: the
same iteration counts (within one step) and the same solutions; the lockstep
run launches fewer kernels. Two families: a well-conditioned 6^3 one whose
hierarchies line up (solutions to 1e-9 relative), and the SI 18^3 one whose
level counts differ between subspaces and between frequencies (cond ~ 1e10:
solutions to 1e-6 relative, the bar the oracle parity tests use for these
systems). The switch is read once per process, so each run is a child
process."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {pkg!r})
import sparsesolv_ngsolve as ss
from sparsesolv_ngsolve import hcurl as H
d = H.eddy_family({nc}, freqs={freqs!r}, nrhs=4, **{kw!r})
pres = [ss.ComplexCompactAMSPreconditioner(a, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                           coord_y=d["coords"][1], coord_z=d["coords"][2]) for a in d["a_real"]]
lv = [[len(p.levels(k)) for k in range(4)] for p in pres]
bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=1000,
                          tol={tol!r})
X = bs.Solve(d["B"])
print(json.dumps(dict(levels=lv, its=bs.iterations.tolist(), launches=int(bs.last_timing["kernel_launches"]),
                      x=np.asarray(X).view(np.float64).ravel().tolist())))
"""


FAMILIES = {
    "aligned": dict(nc=6, freqs=[1e2, 1e3, 1e4, 3e4], kw=dict(nu_r_core=1.0, mass_eps=1.0, sigma=1e5), tol=1e-10,
                    rtol=1e-9),
    "ragged": dict(nc=18, freqs=[1e3, 1e4, 1e5], kw={}, tol=1e-8, rtol=1e-6),
}


def _run(env_value, fam):
    env = dict(os.environ)
    env["SSV_AMS_MULTI"] = env_value
    code = CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "ngsolve-sparsesolv_b200"), nc=fam["nc"],
                        freqs=fam["freqs"], kw=fam["kw"], tol=fam["tol"])
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("family", sorted(FAMILIES))
def test_lockstep_preconditioners_match_branches(family):
    fam = FAMILIES[family]
    lock = _run("1", fam)
    br = _run("0", fam)
    lv = lock["levels"]
    aligned = all(l[0] == lv[0][0] and l[1:] == [lv[0][1]] * 3 for l in lv)
    assert aligned == (family == "aligned"), lv
    assert lock["launches"] < br["launches"]
    a, b = np.array(lock["its"]), np.array(br["its"])
    assert (np.abs(a - b) <= 1).all(), (a, b)
    xa, xb = np.array(lock["x"]), np.array(br["x"])
    assert np.abs(xa - xb).max() <= fam["rtol"] * np.abs(xb).max()
