"""Serving layer: results checked against the CPU oracle's operator, the same
result alone and in a concurrent mix, and admission by HBM budget.

Every request solves M x = b on the odd checkerboard to a relative FP64
true residual of 1e-10 (mixed precision, reliable updates).  Its result
must satisfy |b - M x| / |b| <= 1e-9 with M the oracle's FP64 operator
(built from the host clover term, which matches the device construction),
and a request solved alone and in a mix of concurrent requests must agree
to 1e-12 relative L2 (the reductions have a fixed order, so in practice
the two are bitwise equal).
"""
import numpy as np
import pytest

from helpers import rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu

VOLS = [(4, 4, 4, 8), (8, 4, 4, 8)]
MU = 0.05
CSW = 1.0


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def gauges():
    return {d: F.make_gauge(d, 21 + i, "exp", eps=0.3) for i, d in enumerate(VOLS)}


def _requests():
    """(volume, kind, kappa, nrhs, seed) of a small mixed workload."""
    out = []
    kinds = ["wilson", "clover", "tm", "tmclover"]
    rng = np.random.default_rng(5)
    for i in range(8):
        out.append((VOLS[i % 2], kinds[i % 4], float(rng.uniform(0.115, 0.125)), 1 + i % 3, 100 + i))
    return out


def _rhs(dims, nrhs, seed):
    return np.stack([F.gaussian_spinor(dims, seed + k) for k in range(nrhs)])


def _oracle_op(oracle, dims, gauge, kind, mass):
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    if kind in ("wilson", "tm"):
        return oracle.OracleOp(kind, L, gauge, mass=mass, twisted_mass=MU if kind == "tm" else 0.0)
    cl = F.make_clover(dims, gauge, mass, CSW)
    if kind == "clover":
        return oracle.OracleOp(kind, L, gauge, clov=cl[1], invclov=F.invert_clover(cl[0]), mass=mass)
    return oracle.OracleOp(kind, L, gauge, clov=cl[1], finv=F.twisted_full_inverse(cl[0], MU), mass=mass,
                           rho=MU)


def _serve(api, gauges, reqs, slots, budget=8 << 30, **kw):
    srv = api.Server(budget, slots=slots, low_prec="f16", **kw)
    ens = {d: srv.add_ensemble(d, g) for d, g in gauges.items()}
    results = []
    if slots == 1:
        for d, kind, kappa, nrhs, seed in reqs:
            t = srv.submit(ens[d], kind, _rhs(d, nrhs, seed), F.kappa_to_mass(kappa), CSW, MU)
            results.append(srv.wait(t))
    else:
        tickets = [srv.submit(ens[d], kind, _rhs(d, nrhs, seed), F.kappa_to_mass(kappa), CSW, MU)
                   for d, kind, kappa, nrhs, seed in reqs]
        results = [srv.wait(t) for t in tickets]
    stats = srv.stats()
    srv.close()
    return results, stats


def test_serve_results_match_oracle(api, oracle, gauges):
    reqs = _requests()
    results, stats = _serve(api, gauges, reqs, slots=3)
    assert stats["completed"] == len(reqs) and stats["failed"] == 0
    for (d, kind, kappa, nrhs, seed), (x, info) in zip(reqs, results):
        assert info["status"] == 0 and info["true_rel_resid"] < 1e-10, (kind, info)
        op = _oracle_op(oracle, d, gauges[d], kind, F.kappa_to_mass(kappa))
        b = _rhs(d, nrhs, seed)
        for k in range(nrhs):
            r = b[k] - op.apply(x[k], 1, 1)
            assert np.linalg.norm(r) / np.linalg.norm(b[k]) < 1e-9, (kind, k)
        assert info["latency_s"] >= info["solve_s"] > 0


def test_serve_richardson_matches_oracle(api, oracle, gauges):
    """The server with the InvRichardsonMultiPrec solver (FP64 defect
    correction, BiCGStab inner on the low-precision operator)."""
    reqs = _requests()
    results, stats = _serve(api, gauges, reqs, slots=3, solver="richardson", delta=0.005)
    assert stats["completed"] == len(reqs) and stats["failed"] == 0
    for (d, kind, kappa, nrhs, seed), (x, info) in zip(reqs, results):
        assert info["status"] == 0 and info["true_rel_resid"] < 1e-10, (kind, info)
        op = _oracle_op(oracle, d, gauges[d], kind, F.kappa_to_mass(kappa))
        b = _rhs(d, nrhs, seed)
        for k in range(nrhs):
            r = b[k] - op.apply(x[k], 1, 1)
            assert np.linalg.norm(r) / np.linalg.norm(b[k]) < 1e-9, (kind, k)


def test_serve_same_alone_and_in_mix(api, gauges):
    reqs = _requests()
    alone, _ = _serve(api, gauges, reqs, slots=1)
    mixed, stats = _serve(api, gauges, reqs, slots=4)
    assert stats["running_peak"] >= 2, stats
    bitwise = True
    for (xa, ia), (xm, im) in zip(alone, mixed):
        assert rel_l2(xm, xa) <= 1e-12
        bitwise = bitwise and np.array_equal(xa, xm)
        assert ia["n_iters"] == im["n_iters"]
    print("alone == mix bitwise:", bitwise)


def test_serve_admission_by_budget(api, gauges):
    d = VOLS[1]
    probe = api.Server(8 << 30, slots=1)
    e = probe.add_ensemble(d, gauges[d])
    resident = probe.stats()["resident_bytes"]
    b = _rhs(d, 2, 7)
    need = probe.request_bytes(e, "clover", b)
    probe.close()
    # room for one such request at a time, with four slots
    srv = api.Server(resident + need + need // 2, slots=4)
    e = srv.add_ensemble(d, gauges[d])
    ts = [srv.submit(e, "clover", b, F.kappa_to_mass(0.12)) for _ in range(3)]
    outs = [srv.wait(t) for t in ts]
    st = srv.stats()
    assert st["running_peak"] == 1 and st["completed"] == 3, st
    assert st["reserved_peak_bytes"] <= resident + need + need // 2 - st["resident_bytes"] + need
    for x, info in outs:
        assert info["status"] == 0 and info["bytes"] == need
    assert rel_l2(outs[1][0], outs[0][0]) <= 1e-12
    # a request that can never fit is refused at submission
    with pytest.raises(Exception):
        srv.submit(e, "clover", _rhs(d, 8, 9), F.kappa_to_mass(0.12))
    srv.close()
