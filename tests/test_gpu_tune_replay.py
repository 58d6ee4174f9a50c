"""AMS shape-tuner record and replay (SSV_AMS_TUNE_SAVE / SSV_AMS_TUNE_LOAD):
a run that replays the choices recorded by an earlier run uses the same
launch shapes, so its PCG solve is bitwise equal to the recording run's (the
reductions are deterministic); a file recorded on another matrix stops the
replay at the first entry that names a different matrix, says so on stderr,
and the tuner times from there on (the solve still converges). Each run is a
child process, since the switches are read once per process."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "tests", "host", "_build")

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {pkg!r})
import sparsesolv_ngsolve as ss
from sparsesolv_ngsolve import hcurl as H
d = H.magnetostatic({nc})
p = ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                coord_y=d["coords"][1], coord_z=d["coords"][2])
inv = ss.PCGSolver(d["A"], p, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
x = np.zeros(d["A"].shape[0])
r = inv.Solve(d["f"], x)
print(json.dumps(dict(conv=bool(r.converged), its=int(r.iterations), x=x.tolist())))
"""


def _run(nc, **env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    code = CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "ngsolve-sparsesolv_b200"), nc=nc)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), r.stderr


def test_replay_reproduces_recorded_shapes():
    os.makedirs(OUT, exist_ok=True)
    f = os.path.join(OUT, "tune_mag10.txt")
    if os.path.exists(f):
        os.remove(f)
    rec, _ = _run(10, SSV_AMS_TUNE_SAVE=f)
    lines = open(f).read().split("\n")
    assert any(l.startswith("csr ") for l in lines) and any(l.startswith("pi ") for l in lines)
    rep, err = _run(10, SSV_AMS_TUNE_LOAD=f)
    assert "replay stops" not in err, err[-2000:]
    assert rec["conv"] and rep["conv"] and rec["its"] == rep["its"]
    assert np.array_equal(np.array(rec["x"]), np.array(rep["x"]))
    other, err = _run(8, SSV_AMS_TUNE_LOAD=f)  # recorded on the 10^3 matrices
    assert "replay stops" in err, err[-2000:]
    assert other["conv"]
