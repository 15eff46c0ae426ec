"""Unpreconditioned solves through an even-odd solver
(include/qphix/unprec_solver_wrapper.h:17-99 with the AbstractUnprecSolver
driver of include/qphix/abs_solver.h), Python form, against the CPU oracle.

The full clover operator is [[A_ee, -D_eo/2], [-D_oe/2, A_oo]] (the Wilson
operator has A = 4 + m); isign = -1 uses the daggered hops.  For each
solve checkerboard and isign the wrapper's solution meets the target on the
FULL residual (recomputed with the oracle's Dslash and clover term), and
equals the oracle's own prepare / BiCGStab / reconstruct chain to 1e-8.
The twisted-mass operators have no M_offdiag (as in the reference) and the
wrapper refuses them.
"""
import numpy as np
import pytest

from helpers import make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu
MASS = 0.1


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def setup():
    return make_setup((4, 4, 4, 8), seed=41, gauge_kind="weak", mass=MASS, mu=0.1)


def _full_residual(oracle, L, s, diag, x, b, isign):
    """|| M_full x - b || / || b || with diag(v, cb) the diagonal block"""
    r = [diag(x[cb], cb) - 0.5 * oracle.dslash(L, x[1 - cb], s["gauge"], isign, cb) - b[cb]
         for cb in (0, 1)]
    return np.sqrt(sum(np.linalg.norm(v) ** 2 for v in r) / sum(np.linalg.norm(v) ** 2 for v in b))


def _oracle_unprec(oracle, L, s, O, diag_inv, b, isign, solve_cb):
    o = 1 - solve_cb
    bp = b[solve_cb] + 0.5 * oracle.dslash(L, diag_inv(b[o]), s["gauge"], isign, solve_cb)
    xs, _ = oracle.bicgstab(O, bp, 1e-10, 2000, isign, solve_cb)
    xo = diag_inv(b[o] + 0.5 * oracle.dslash(L, xs, s["gauge"], isign, o))
    return (xo, xs) if solve_cb == 1 else (xs, xo)


@pytest.mark.parametrize("solve_cb", [1, 0])
@pytest.mark.parametrize("isign", [1, -1])
def test_unprec_clover(api, oracle, setup, solve_cb, isign):
    s = setup
    dims = s["dims"]
    o = 1 - solve_cb
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 12).upload(s["gauge"])
    # the even-odd operator on solve_cb holds A of solve_cb and A^-1 of the other
    A = lat.clover().upload(s["clov"][solve_cb])
    Ainv = lat.clover().upload(s["invclov"][o])
    M = api.EvenOddCloverOperator(u, A, Ainv)
    b = [F.gaussian_spinor(dims, 100 + cb) for cb in (0, 1)]
    fb = api.FullSpinor(lat)
    fx = api.FullSpinor(lat)
    for cb in (0, 1):
        fb.getCBData(cb).upload(b[cb])
    info = api.UnprecSolverWrapper(api.InvBiCGStab(M, 2000), M)(fx, fb, 1e-10, isign, solve_cb)[0]
    assert info["status"] == 0
    x = [fx.getCBData(cb).download() for cb in (0, 1)]
    L = oracle.make_lattice(dims, -1.0)
    assert _full_residual(oracle, L, s, lambda v, cb: oracle.clover_apply(v, s["clov"][cb]), x, b,
                          isign) < 2e-10
    O = oracle.OracleOp("clover", L, s["gauge"], clov=s["clov"][solve_cb], invclov=s["invclov"][o])
    ref = _oracle_unprec(oracle, L, s, O, lambda v: oracle.clover_apply(v, s["invclov"][o]), b, isign,
                         solve_cb)
    assert rel_l2(np.stack(x), np.stack(ref)) < 1e-8


@pytest.mark.parametrize("nrhs", [1, 2])
def test_unprec_wilson(api, oracle, setup, nrhs):
    s = setup
    dims = s["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 12).upload(s["gauge"])
    M = api.EvenOddWilsonOperator(MASS, u)
    b = [np.stack([F.gaussian_spinor(dims, 200 + 2 * k + cb) for k in range(nrhs)]) for cb in (0, 1)]
    fb, fx = api.FullSpinor(lat, nrhs=nrhs), api.FullSpinor(lat, nrhs=nrhs)
    for cb in (0, 1):
        fb.getCBData(cb).upload(b[cb])
    infos = api.UnprecSolverWrapper(api.InvBiCGStab(M, 2000), M)(fx, fb, 1e-10)
    assert len(infos) == nrhs and all(i["status"] == 0 for i in infos)
    L = oracle.make_lattice(dims, -1.0)
    for k in range(nrhs):
        x = [fx.getCBData(cb).download(k) for cb in (0, 1)]
        bk = [b[cb][k] for cb in (0, 1)]
        assert _full_residual(oracle, L, s, lambda v, cb: (4.0 + MASS) * v, x, bk, 1) < 2e-10


def test_unprec_refuses_twisted_mass(api, setup):
    s = setup
    lat = api.Lattice(s["dims"])
    u = lat.gauge("f64", 12).upload(s["gauge"])
    M = api.EvenOddTMWilsonOperator(MASS, 0.1, u)
    fb, fx = api.FullSpinor(lat), api.FullSpinor(lat)
    with pytest.raises(NotImplementedError):
        api.UnprecSolverWrapper(api.InvBiCGStab(M, 100), M)(fx, fb, 1e-10)
