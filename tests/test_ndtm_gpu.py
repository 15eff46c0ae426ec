"""Two-flavour (non-degenerate) twisted-mass Wilson operator and its CG solve
through the C ABI against the CPU oracle
(include/qphix/ndtm_reuse_operator.h:16-110).

A two-flavour field holds (up, down) pairs as right-hand sides 2k, 2k + 1.
Operator: relative L2 within the stated tolerance of each storage precision
(FP64 1e-13, FP32 1e-6, FP16 4e-3, Q16 1e-3) for every isign and target
checkerboard, one and two doublets per field.  CG on M^+ M treats each pair
as one system whose inner products sum over both flavours (the reference's
num_flav = 2 solver): FP64 iteration counts equal the oracle's two-flavour
CG, and the true residual, recomputed with the oracle, meets the target.
"""
import numpy as np
import pytest

from helpers import TOL, make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu

MASS, MU, EPS = 0.1, 0.3, 0.2


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def setup():
    return make_setup((4, 4, 4, 8), seed=21, gauge_kind="weak", mass=MASS, mu=0.1)


def _doublets(dims, n, seed):
    return [np.stack([F.gaussian_spinor(dims, seed + 2 * k), F.gaussian_spinor(dims, seed + 2 * k + 1)])
            for k in range(n)]


@pytest.mark.parametrize("prec", ["f64", "f32", "f16", "q16"])
@pytest.mark.parametrize("ndoub", [1, 2])
def test_ndtm_operator(api, oracle, setup, prec, ndoub):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, 12).upload(setup["gauge"])
    M = api.EvenOddNDTMWilsonOperator(MASS, MU, EPS, u)
    L = oracle.make_lattice(dims, -1.0)
    O = oracle.OracleOp("ndtm", L, setup["gauge"], mass=MASS, twisted_mass=MU, epsilon=EPS)
    ds = _doublets(dims, ndoub, 60)
    x = lat.spinor(prec, 2 * ndoub).upload(np.concatenate(ds))
    y = lat.spinor(prec, 2 * ndoub)
    for isign in (1, -1):
        for cb in (0, 1):
            M(y, x, isign, cb)
            out = y.download()
            for k in range(ndoub):
                ref = O.apply(ds[k], isign, cb)
                assert rel_l2(out[2 * k:2 * k + 2], ref) < TOL[prec], (prec, isign, cb, k)


def test_ndtm_cg(api, oracle, setup):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 12).upload(setup["gauge"])
    M = api.EvenOddNDTMWilsonOperator(MASS, MU, EPS, u)
    L = oracle.make_lattice(dims, -1.0)
    O = oracle.OracleOp("ndtm", L, setup["gauge"], mass=MASS, twisted_mass=MU, epsilon=EPS)
    ds = _doublets(dims, 2, 80)
    b = lat.spinor("f64", 4).upload(np.concatenate(ds))
    x = lat.spinor("f64", 4)
    infos = api.InvCG(M, 2000)(x, b, 1e-10)
    xs = x.download()
    for k in range(2):
        xo, io = oracle.cg(O, ds[k], 1e-10, 2000)
        xk = xs[2 * k:2 * k + 2]
        assert infos[2 * k]["n_iters"] == infos[2 * k + 1]["n_iters"] == io.n_iters, (infos[2 * k], io.n_iters)
        assert rel_l2(xk, xo) < 1e-8
        r = ds[k] - O.apply(O.apply(xk, 1), -1)
        assert np.linalg.norm(r) / np.linalg.norm(ds[k]) < 1e-10
        assert infos[2 * k]["true_rel_resid"] < 1e-10 and infos[2 * k]["status"] == 0


def test_ndtm_other_solvers_refuse(api, setup):
    """Only CG solves two-flavour systems (as one coupled pair)."""
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 12).upload(setup["gauge"])
    M = api.EvenOddNDTMWilsonOperator(MASS, MU, EPS, u)
    b = lat.spinor("f64", 2).upload(np.concatenate(_doublets(dims, 1, 90)))
    x = lat.spinor("f64", 2)
    with pytest.raises(Exception):
        api.InvBiCGStab(M, 100)(x, b, 1e-10)
