"""The one-launch IC sweep (SSV_IC_SWEEP=one: every colour of a triangular
solve in one launch, work units in ticket order, bounded waits on per-colour
completion counters) computes exactly what the per-colour launches compute:
same per-row arithmetic in the same order, so ICCG iterations, residual
histories and solutions are bitwise equal. The switch is read once per
process, so the one-launch solve runs in a child process."""
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
from sparsesolv_ngsolve import problems as P
out = {{}}
for n, bs, cplx in ((24, 4, False), (16, 8, False), (12, 4, True)):
    A = P.laplacian_7pt(n)
    b = P.random_rhs(A.shape[0], 0)
    if cplx:
        A = P.complex_shifted(A, 0.2 + 0.1j)
        b = b + 0.5j * b[::-1]
    fd = P.boundary_freedofs_7pt(n)
    s = ss.SparseSolvSolver(A, method="ICCG", freedofs=fd, tol=1e-10, use_abmc=True, abmc_block_size=bs,
                            save_residual_history=True)
    x = np.zeros_like(b)
    r = s.Solve(b, x)
    out[f"{{n}}_{{bs}}_{{int(cplx)}}"] = dict(it=int(r.iterations), hist=[float(h) for h in r.residual_history],
                                         x=np.asarray(x).view(np.float64).tolist())
print(json.dumps(out))
"""


def _run(env_value):
    env = dict(os.environ)
    if env_value is None:
        env.pop("SSV_IC_SWEEP", None)
    else:
        env["SSV_IC_SWEEP"] = env_value
    code = CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "ngsolve-sparsesolv_b200"))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_one_launch_sweep_matches_per_colour_launches():
    per_colour = _run(None)
    one = _run("one")
    assert per_colour.keys() == one.keys()
    for k in per_colour:
        a, b = per_colour[k], one[k]
        assert a["it"] == b["it"], k
        assert a["hist"] == b["hist"], k
        assert np.array_equal(np.array(a["x"]), np.array(b["x"])), k
