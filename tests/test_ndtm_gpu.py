"""Two-flavour (non-degenerate) twisted-mass Wilson and clover operators and
their CG solves through the C ABI against the CPU oracle
(include/qphix/ndtm_reuse_operator.h:16-110,
include/qphix/ndtm_reuse_operator_clover.h:23-165).  For the clover operator
also the device-built two-flavour inverse fields (against numpy, 1e-13) and
the fused two-flavour hop + inverse clover term.

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


# ---------------------------------------------------------------------------
# two-flavour twisted-mass clover (include/qphix/ndtm_reuse_operator_clover.h)
# ---------------------------------------------------------------------------
NDC_TOL = {"f64": 1e-13, "f32": 1e-6, "f16": 4e-3, "q16": 1e-3}


def _ndc_fields(api, lat, setup, prec, target_cb, mu, eps):
    """A of target_cb and the device-built inverses of the other checkerboard"""
    A = lat.clover(prec).upload(setup["clov"][target_cb])
    A_other = lat.clover("f64").upload(setup["clov"][1 - target_cb])
    fu, fd, c = lat.full_clover(prec), lat.full_clover(prec), lat.clover(prec)
    api.clover_invert_ndtm(fu, fd, c, A_other, mu, eps)
    return A, (fu, fd), c


def test_ndtm_clover_inverse_build(api, setup):
    lat = api.Lattice(setup["dims"])
    A = lat.clover("f64").upload(setup["clov"][0])
    fu, fd, c = lat.full_clover(), lat.full_clover(), lat.clover()
    api.clover_invert_ndtm(fu, fd, c, A, MU, EPS)
    hu, hd, hc = F.ndtm_clover_inverses(setup["clov"][0], MU, EPS)
    assert rel_l2(fu.download(), F.full_clover_to_real(hu).reshape(-1, 144)) < 1e-13
    assert rel_l2(fd.download(), F.full_clover_to_real(hd).reshape(-1, 144)) < 1e-13
    assert rel_l2(c.download(), hc.reshape(-1, 72)) < 1e-13


@pytest.mark.parametrize("prec", ["f64", "f32", "f16", "q16"])
@pytest.mark.parametrize("ndoub", [1, 2])
def test_ndtm_clover_operator(api, oracle, setup, prec, ndoub):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, 12).upload(setup["gauge"])
    L = oracle.make_lattice(dims, -1.0)
    ds = _doublets(dims, ndoub, 160)
    x = lat.spinor(prec, 2 * ndoub).upload(np.concatenate(ds))
    y = lat.spinor(prec, 2 * ndoub)
    for cb in (0, 1):
        A, finv, c = _ndc_fields(api, lat, setup, prec, cb, MU, EPS)
        M = api.EvenOddNDTMCloverOperator(MU, EPS, u, A, c, finv)
        hu, hd, hc = F.ndtm_clover_inverses(setup["clov"][1 - cb], MU, EPS)
        O = oracle.OracleOp("ndtmclover", L, setup["gauge"], clov=setup["clov"][cb], invclov=hc, finv=(hu, hd),
                            twisted_mass=MU, epsilon=EPS)
        for isign in (1, -1):
            M(y, x, isign, cb)
            out = y.download()
            for k in range(ndoub):
                ref = O.apply(ds[k], isign, cb)
                assert rel_l2(out[2 * k:2 * k + 2], ref) < NDC_TOL[prec], (prec, isign, cb, k)


def test_ndtm_clover_two_flavour_hop(api, oracle, setup):
    """qphix_gpu_dslash_two_flav_clover = Wilson hop of both flavours, then
    u_up = F_a t_up + C t_dn, u_dn = F_b t_dn + C t_up (F swapped for isign = -1)"""
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 18).upload(setup["gauge"])
    A = lat.clover("f64").upload(setup["clov"][0])
    fu, fd, c = lat.full_clover(), lat.full_clover(), lat.clover()
    api.clover_invert_ndtm(fu, fd, c, A, MU, EPS)
    hu, hd, hc = F.ndtm_clover_inverses(setup["clov"][0], MU, EPS)
    D = api.TMClovDslashTwoFlav(lat, -1.0, 1.0, 1.0, MU, EPS)
    d = _doublets(dims, 1, 170)[0]
    x = lat.spinor("f64", 2).upload(d)
    y = lat.spinor("f64", 2)
    L = oracle.make_lattice(dims, -1.0)
    for isign in (1, -1):
        D.dslash_inverse_clover(y, x, u, (fu, fd), c, isign, 0)
        t = [oracle.dslash(L, d[f], setup["gauge"], isign, 0) for f in (0, 1)]
        fa, fb = (hu, hd) if isign == 1 else (hd, hu)
        ref = np.stack([oracle.fullclover_apply(t[0], fa) + oracle.clover_apply(t[1], hc),
                        oracle.fullclover_apply(t[1], fb) + oracle.clover_apply(t[0], hc)])
        assert rel_l2(y.download(), ref) < 1e-13


def test_ndtm_clover_cg(api, oracle, setup):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 12).upload(setup["gauge"])
    A, finv, c = _ndc_fields(api, lat, setup, "f64", 1, MU, EPS)
    M = api.EvenOddNDTMCloverOperator(MU, EPS, u, A, c, finv)
    hu, hd, hc = F.ndtm_clover_inverses(setup["clov"][0], MU, EPS)
    L = oracle.make_lattice(dims, -1.0)
    O = oracle.OracleOp("ndtmclover", L, setup["gauge"], clov=setup["clov"][1], invclov=hc, finv=(hu, hd),
                        twisted_mass=MU, epsilon=EPS)
    ds = _doublets(dims, 2, 180)
    b = lat.spinor("f64", 4).upload(np.concatenate(ds))
    x = lat.spinor("f64", 4)
    infos = api.InvCG(M, 2000)(x, b, 1e-10)
    xs = x.download()
    for k in range(2):
        xo, io = oracle.cg(O, ds[k], 1e-10, 2000)
        xk = xs[2 * k:2 * k + 2]
        assert infos[2 * k]["n_iters"] == infos[2 * k + 1]["n_iters"] == io.n_iters, (infos[2 * k], io.n_iters)
        r = ds[k] - O.apply(O.apply(xk, 1), -1)
        assert np.linalg.norm(r) / np.linalg.norm(ds[k]) < 1e-10
