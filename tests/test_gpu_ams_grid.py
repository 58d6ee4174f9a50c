"""Whole AMS V-cycles as single cooperative launches (SSV_AMS_GRID=1): the
gradient V-cycle and the three nodal V-cycles each run as one launch with
grid-wide barriers instead of a chain of per-level launches. Inside Krylov
solves they must reproduce the oracle's solves as the chain does: PCG (FP64
and FP32 hierarchies) and COCR with the complex form, on a ragged-hierarchy
system too, in both graph modes (the default WHILE-conditional graph and
host-relaunched chunks), with fewer kernel launches than the chain. The
switch is read when the work vectors are set up, so each mode runs in a
child process; the same child with SSV_AMS_GRID=0 gives the chain's launch
count."""
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
from oracle import oracle as O
out = {{}}

def ams(d, mat, **kw):
    return ss.CompactAMSPreconditioner(mat, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                       coord_y=d["coords"][1], coord_z=d["coords"][2], **kw)

for name, d, prec in [("mag_well", H.magnetostatic(8, nu_iron=1.0, mass_eps=1.0), "fp64"),
                      ("mag_well32", H.magnetostatic(8, nu_iron=1.0, mass_eps=1.0), "fp32"),
                      ("mag_si", H.magnetostatic(10), "fp64")]:
    p = ams(d, d["A"], precision=prec)
    inv = ss.PCGSolver(d["A"], p, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    x = np.zeros(d["A"].shape[0])
    r = inv.Solve(d["f"], x)
    o = O.AmsOracle(d["A"], d["G"], d["freedofs"], *d["coords"])
    xo, ro, _ = o.pcg(d["f"], config=O.default_config(tolerance=1e-10, max_iterations=500))
    fd = d["freedofs"].astype(bool)
    res = np.linalg.norm((d["f"] - d["A"] @ np.where(fd, x, 0))[fd]) / np.linalg.norm(d["f"])
    out[name] = dict(conv=bool(r.converged), its=int(r.iterations), its_o=int(ro.iterations),
                     x=float(np.abs(x - xo).max() / np.abs(xo).max()), res=float(res),
                     launches=int(r.kernel_launches))

for name, d in [("eddy_well", H.eddy_current(8, nu_r_core=1.0, mass_eps=1.0, sigma=1e5, freq=1e3)),
                ("eddy_ragged", H.eddy_current(18, freq=1e3, nu_r_core=0.1, mass_eps=1.0))]:
    p = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                           coord_y=d["coords"][1], coord_z=d["coords"][2])
    inv = ss.COCRSolver(d["A"], p, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    x = inv * d["f"]
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    xo, it, _ = o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    out[name] = dict(its=int(inv.iterations), its_o=int(it), x=float(np.abs(x - xo).max() / np.abs(xo).max()),
                     levels=[len(p.levels(s)) for s in range(4)])
print(json.dumps(out))
"""


def _run(grid, graph_mode=None):
    env = dict(os.environ)
    env["SSV_AMS_GRID"] = grid
    if graph_mode:
        env["SSV_GRAPH_MODE"] = graph_mode
    code = CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "ngsolve-sparsesolv_b200"))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def chain():
    return _run("0")


@pytest.mark.parametrize("graph_mode", ["while", "chunk"])
def test_grid_vcycles_match_oracle(graph_mode, chain):
    out = _run("1", graph_mode)
    for name, xtol in [("mag_well", 1e-8), ("mag_si", 1e-6)]:
        c = out[name]
        assert c["conv"] and c["res"] <= 1e-10 * 1.01, (name, c)
        assert abs(c["its"] - c["its_o"]) <= max(1, int(0.02 * c["its_o"])), (name, c)
        assert c["x"] <= xtol, (name, c)
    c = out["mag_well32"]  # FP32 hierarchies: FP64 outer recurrence, iteration bound of the FP32 form
    assert c["conv"] and c["res"] <= 1e-10 * 1.01 and c["its"] <= 1.5 * out["mag_well"]["its_o"] + 2, c
    for name in ("eddy_well", "eddy_ragged"):
        c = out[name]
        assert abs(c["its"] - c["its_o"]) <= max(1, int(0.02 * c["its_o"])), (name, c)
        assert c["x"] <= 1e-8, (name, c)
    assert len(set(out["eddy_ragged"]["levels"][1:])) > 1, out["eddy_ragged"]["levels"]
    for name in ("mag_well", "mag_si"):  # one launch per V-cycle instead of a per-level chain
        per_it = out[name]["launches"] / max(out[name]["its"], 1)
        per_it_chain = chain[name]["launches"] / max(chain[name]["its"], 1)
        assert per_it < per_it_chain, (name, per_it, per_it_chain)
