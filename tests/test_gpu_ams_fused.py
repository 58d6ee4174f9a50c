"""V-cycles through the fused level products (SSV_AMS_FUSED=1, the default for
every FP64 hierarchy and for the FP32 nodal ones: b' = R b down, x = U [b; e]
up, two launches per level, and below 2048 rows the dense tail where the
coarsest factors allow one) against the four per-level passes
(SSV_AMS_FUSED=0): the same PCG and COCR iteration counts (within one step)
and solutions, fewer kernel launches per iteration -- in the FP64 form and in
the FP32 form (fused nodal hierarchies, the gradient one in four passes in
both runs). The ragged-hierarchy system checks the lockstep form with
hierarchies of different depths. The switch is read at set-up, so each mode
runs in a child process."""
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
out = {{}}
for name, d in [("mag_well", H.magnetostatic(10, nu_iron=1.0, mass_eps=1.0)), ("mag_si", H.magnetostatic(10))]:
    p = ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                    coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.PCGSolver(d["A"], p, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    x = np.zeros(d["A"].shape[0])
    r = inv.Solve(d["f"], x)
    out[name] = dict(conv=bool(r.converged), its=int(r.iterations), launches=int(r.kernel_launches), x=x.tolist())
    p.precision = "fp32"
    x = np.zeros(d["A"].shape[0])
    r = inv.Solve(d["f"], x)
    out[name + "_fp32"] = dict(conv=bool(r.converged), its=int(r.iterations), launches=int(r.kernel_launches))
d = H.eddy_current(18, freq=1e3, nu_r_core=0.1, mass_eps=1.0)
p = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                       coord_y=d["coords"][1], coord_z=d["coords"][2])
inv = ss.COCRSolver(d["A"], p, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
x = inv * d["f"]
out["eddy_ragged"] = dict(its=int(inv.iterations), x=np.asarray(x).view(np.float64).tolist(),
                          levels=[len(p.levels(s)) for s in range(4)])
print(json.dumps(out))
"""


def _run(fused):
    env = dict(os.environ)
    env["SSV_AMS_FUSED"] = fused
    code = CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "ngsolve-sparsesolv_b200"))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_fused_vcycles_match_four_pass_form():
    fu, four = _run("1"), _run("0")
    for name, xtol in [("mag_well", 1e-9), ("mag_si", 1e-6)]:
        a, b = fu[name], four[name]
        assert a["conv"] and b["conv"], name
        assert abs(a["its"] - b["its"]) <= 1, (name, a["its"], b["its"])
        xa, xb = np.array(a["x"]), np.array(b["x"])
        assert np.abs(xa - xb).max() <= xtol * np.abs(xb).max(), name
        assert a["launches"] / a["its"] < b["launches"] / b["its"], name
    for name in ("mag_well_fp32", "mag_si_fp32"):
        a, b = fu[name], four[name]
        assert a["conv"] and b["conv"], name
        assert abs(a["its"] - b["its"]) <= 1, (name, a["its"], b["its"])
        assert a["launches"] / a["its"] < b["launches"] / b["its"], name
    a, b = fu["eddy_ragged"], four["eddy_ragged"]
    assert len(set(a["levels"][1:])) > 1, a["levels"]
    assert abs(a["its"] - b["its"]) <= 1, (a["its"], b["its"])
    xa, xb = np.array(a["x"]), np.array(b["x"])
    assert np.abs(xa - xb).max() <= 1e-9 * np.abs(xb).max()
