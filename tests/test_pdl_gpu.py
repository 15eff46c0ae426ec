"""Programmatic dependent launch (launch_pdl, qpx_common.cuh) changes when the
Dslash, BLAS and fold kernels start, not what they compute: a BiCGStab solve
on 16^3x32, whose launches are above the attribute's block threshold, takes
the same iterations and gives a bit-identical solution with the attribute
(the default) and without it (QPHIX_GPU_PDL=0, which the library reads once
per process, hence two child processes)."""
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
sys.path.insert(0, sys.argv[2])
from qphix_b200 import api, fields as F
dims = (16, 16, 16, 32)
g = F.make_gauge(dims, 91, "exp", eps=0.3)
cl = F.make_clover(dims, g, -0.2, 1.0)
lat = api.Lattice(dims)
u = lat.gauge("f32", 12).upload(g)
M = api.EvenOddCloverOperator(u, lat.clover("f32").upload(cl[1]),
                              lat.clover("f32").upload(F.invert_clover(cl[0])))
b = lat.spinor("f32").upload(F.gaussian_spinor(dims, 92))
x = lat.spinor("f32")
info = api.InvBiCGStab(M, 2000)(x, b, 1e-6)[0]
np.save(sys.argv[1], x.download())
print(json.dumps({"n_iters": info["n_iters"], "status": info["status"], "launches": api.launch_count()}))
"""


def _run(tmp_path, tag, pdl):
    env = dict(os.environ)
    if pdl:
        env.pop("QPHIX_GPU_PDL", None)
    else:
        env["QPHIX_GPU_PDL"] = "0"
    out = str(tmp_path / f"x_{tag}.npy")
    r = subprocess.run([sys.executable, "-c", CHILD, out, ROOT], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(out)


def test_pdl_does_not_change_results(tmp_path):
    a, xa = _run(tmp_path, "pdl", True)
    b, xb = _run(tmp_path, "plain", False)
    assert a["status"] == 0 and b["status"] == 0
    assert a["n_iters"] == b["n_iters"]
    assert np.array_equal(xa, xb)
