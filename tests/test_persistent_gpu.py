"""Persistent-kernel CG (qphix_b200/csrc/qpx_persist.cuh): the whole
iteration loop of InvCG (include/qphix/invcg.h:281-417) in one cooperative
launch, for small lattices.

Checked against the CPU oracle (FP64: the oracle's iteration count, the
solution to 1e-8 and the true residual |b - M^+ M x| / |b| recomputed in
FP64) and against the graph-captured iterations of the regular path
(QPHIX_GPU_PERSISTENT=0): the persistent kernel runs the same Dslash block
code, folds the reductions in the same order and runs the same finalize, so
both paths take the same number of iterations and reach the same solution.
The launch counter shows which path ran: a persistent solve is a handful of
launches, the graph path hundreds.
"""
import numpy as np
import pytest

from helpers import make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


def _ops(api, oracle, s, kind, prec, recon):
    dims = s["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, recon).upload(s["gauge"])
    Lg = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    keep = [u]
    if kind == "wilson":
        M = api.EvenOddWilsonOperator(s["mass"], u)
        O = oracle.OracleOp("wilson", Lg, s["gauge"], mass=s["mass"])
    else:
        A = lat.clover(prec).upload(s["clov"][1])
        Ai = lat.clover(prec).upload(s["invclov"][0])
        keep += [A, Ai]
        M = api.EvenOddCloverOperator(u, A, Ai)
        O = oracle.OracleOp("clover", Lg, s["gauge"], clov=s["clov"][1], invclov=s["invclov"][0])
    return lat, M, O, keep


def _solve(api, lat, M, b, prec, mode, monkeypatch, rsd=1e-10, max_iters=500):
    monkeypatch.setenv("QPHIX_GPU_PERSISTENT", mode)
    nrhs = b.shape[0] if b.ndim == 4 else 1
    gx, gb = lat.spinor(prec, nrhs), lat.spinor(prec, nrhs).upload(b)
    n0 = api.launch_count()
    info = api.InvCG(M, max_iters)(gx, gb, rsd)
    return gx.download(), info, api.launch_count() - n0


@pytest.mark.parametrize("kind,recon", [("wilson", 12), ("wilson", 18), ("clover", 12), ("clover", 18)])
def test_persistent_cg_fp64_vs_oracle(api, oracle, kind, recon, monkeypatch):
    dims = (8, 8, 8, 8)
    s = make_setup(dims, seed=71, gauge_kind="weak", mass=0.1)
    lat, M, O, keep = _ops(api, oracle, s, kind, "f64", recon)
    b = F.gaussian_spinor(dims, 72)
    x, info, nl = _solve(api, lat, M, b, "f64", "1", monkeypatch)
    xo, io = oracle.cg(O, b, 1e-10, 500)
    r = b - O.apply(O.apply(x, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.5e-10
    assert info[0]["status"] == 0 and info[0]["true_rel_resid"] < 1.5e-10
    assert info[0]["n_iters"] == io.n_iters
    assert rel_l2(x, xo) < 1e-8
    assert nl < 40, nl  # one persistent launch plus the set-up and true-residual launches


@pytest.mark.parametrize("prec,nrhs", [("f64", 1), ("f64", 4), ("f32", 1), ("f32", 3)])
def test_persistent_matches_graph_path(api, oracle, prec, nrhs, monkeypatch):
    dims = (4, 4, 8, 8)
    s = make_setup(dims, seed=73, gauge_kind="weak", mass=0.1)
    lat, M, O, keep = _ops(api, oracle, s, "clover", prec, 12)
    b = np.stack([F.gaussian_spinor(dims, 74 + i) for i in range(nrhs)])
    rsd = 1e-10 if prec == "f64" else 1e-5
    xp, ip, np_launch = _solve(api, lat, M, b, prec, "1", monkeypatch, rsd=rsd)
    xg, ig, ng_launch = _solve(api, lat, M, b, prec, "0", monkeypatch, rsd=rsd)
    assert np_launch < ng_launch
    xp, xg = xp.reshape(nrhs, -1), xg.reshape(nrhs, -1)
    for i in range(nrhs):
        assert ip[i]["n_iters"] == ig[i]["n_iters"]
        assert ip[i]["status"] == 0
        assert ip[i]["true_rel_resid"] < 1.5 * rsd
        assert rel_l2(xp[i], xg[i]) < (1e-12 if prec == "f64" else 1e-5)


def test_persistent_max_iters_and_restart(api, oracle, monkeypatch):
    """max_iters stops the persistent loop as it stops the graph path (status
    1, the same iterate), and a second solve on the same lattice reuses the
    barrier from a clean state."""
    dims = (8, 8, 8, 8)
    s = make_setup(dims, seed=75, gauge_kind="weak", mass=0.05)
    lat, M, O, keep = _ops(api, oracle, s, "wilson", "f64", 12)
    b = F.gaussian_spinor(dims, 76)
    xp, ip, _ = _solve(api, lat, M, b, "f64", "1", monkeypatch, max_iters=7)
    xg, ig, _ = _solve(api, lat, M, b, "f64", "0", monkeypatch, max_iters=7)
    assert ip[0]["status"] == 1 and ig[0]["status"] == 1
    assert ip[0]["n_iters"] == ig[0]["n_iters"]
    assert rel_l2(xp, xg) < 1e-12
    x2, i2, _ = _solve(api, lat, M, b, "f64", "1", monkeypatch)
    assert i2[0]["status"] == 0 and i2[0]["true_rel_resid"] < 1.5e-10


def test_twisted_boundary_falls_back(api, oracle, monkeypatch):
    """A boundary phase needs the general Dslash path, which the persistent
    kernel does not build: the solve runs the graph path and is still right."""
    dims = (4, 4, 4, 8)
    s = make_setup(dims, seed=77, gauge_kind="weak", mass=0.1)
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 12).upload(s["gauge"])
    ph = np.exp(0.3j)
    M = api.EvenOddWilsonOperator(s["mass"], u, use_tbc=[0, 0, 1, 0],
                                  tbc_phases=[[1, 0], [1, 0], [ph.real, ph.imag], [1, 0]])
    Lg = oracle.make_lattice(dims, -1.0, 1.0, 1.0, tbc=[None, None, ph, None])
    O = oracle.OracleOp("wilson", Lg, s["gauge"], mass=s["mass"])
    b = F.gaussian_spinor(dims, 78)
    x, info, nl = _solve(api, lat, M, b, "f64", "1", monkeypatch)
    r = b - O.apply(O.apply(x, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.5e-10
    assert nl > 40  # the graph path ran
