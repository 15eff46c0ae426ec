"""Multi-GPU halo mode (t slabs, qphix_b200/halo.py) emulated on one GPU:
the lattice is cut into 2 or 4 slabs, each on its own lattice object, every
slab packs its boundary faces and reads its neighbours' (LocalSlabs), and
the glued result of the halo Dslash and even-odd operators equals the
whole-lattice oracle: relative L2 <= 1e-13 in FP64, the stated FP16
tolerance in FP16, for both checkerboards and isign, with antiperiodic time
and anisotropic hops; one slab (faces wrapping onto itself) equals the
one-GPU operator bit for bit."""
import ctypes as C

import numpy as np
import pytest

from helpers import TOL, make_setup, rel_l2
from qphix_b200 import _lib as L
from qphix_b200 import fields as F
from qphix_b200 import halo

pytestmark = pytest.mark.gpu
DIMS = (8, 4, 4, 16)
ANISO = (0.9, 1.1)


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def setup():
    return make_setup(DIMS, seed=61, gauge_kind="weak", mass=0.1, mu=0.07)


def _ops(api, ls, s, kind, prec, target_cb):
    p = api.op_params({"wilson": L.WILSON, "clover": L.CLOVER_OP, "tm": L.TM, "tmclover": L.TMCLOVER}[kind],
                      -1.0, ANISO[0], ANISO[1], mass=s["mass"], twisted_mass=s["mu"],
                      prec_mass_rho=s["mu"] if kind == "tmclover" else 0.0)
    other = 1 - target_cb

    def make(slab, lat, exchange):
        u = lat.gauge(prec, 12).upload(slab.cut_gauge(s["gauge"]))
        kw = {}
        if kind == "clover":
            kw = dict(clov=lat.clover(prec).upload(slab.cut_clover(s["clov"][target_cb])),
                      invclov=lat.clover(prec).upload(slab.cut_clover(s["invclov"][other])))
        elif kind == "tmclover":
            f0, f1 = s["finv"][other]
            kw = dict(clov=lat.clover(prec).upload(slab.cut_clover(s["clov"][target_cb])),
                      finv=(lat.full_clover(prec).upload(slab.cut_clover(f0)),
                            lat.full_clover(prec).upload(slab.cut_clover(f1))))
        return halo.SlabOperator(slab, lat, p, u, exchange, **kw)
    return ls.operators(make)


def _oracle_op(oracle, s, kind, target_cb):
    Lg = oracle.make_lattice(DIMS, -1.0, *ANISO)
    other = 1 - target_cb
    if kind == "wilson":
        return oracle.OracleOp("wilson", Lg, s["gauge"], mass=s["mass"])
    if kind == "tm":
        return oracle.OracleOp("tm", Lg, s["gauge"], mass=s["mass"], twisted_mass=s["mu"])
    if kind == "clover":
        return oracle.OracleOp("clover", Lg, s["gauge"], clov=s["clov"][target_cb], invclov=s["invclov"][other])
    return oracle.OracleOp("tmclover", Lg, s["gauge"], clov=s["clov"][target_cb], finv=s["finv"][other],
                           rho=s["mu"])


@pytest.mark.parametrize("nslabs", [2, 4])
@pytest.mark.parametrize("prec", ["f64", "f16"])
def test_halo_wilson_dslash(api, oracle, setup, nslabs, prec):
    s = setup
    ls = halo.LocalSlabs(DIMS, nslabs)
    ops = _ops(api, ls, s, "wilson", prec, 1)
    Lg = oracle.make_lattice(DIMS, -1.0, *ANISO)
    psi = np.stack([F.gaussian_spinor(DIMS, 5), F.gaussian_spinor(DIMS, 6)])
    ins = [lat.spinor(prec, 2).upload(sl.cut_spinor(psi)) for sl, lat in zip(ls.slabs, ls.lats)]
    outs = [lat.spinor(prec, 2) for lat in ls.lats]
    for isign in (1, -1):
        for cb in (0, 1):
            ls.dslash(ops, outs, ins, isign, cb)
            got = np.concatenate([o.download() for o in outs], axis=1)
            for k in range(2):
                ref = oracle.dslash(Lg, psi[k], s["gauge"], isign, cb)
                assert rel_l2(got[k], ref) < TOL[prec], (nslabs, prec, isign, cb, k)


@pytest.mark.parametrize("kind", ["wilson", "clover", "tm", "tmclover"])
@pytest.mark.parametrize("nslabs", [2, 4])
def test_halo_eo_operators(api, oracle, setup, kind, nslabs):
    s = setup
    ls = halo.LocalSlabs(DIMS, nslabs)
    psi = F.gaussian_spinor(DIMS, 7)
    for target_cb in (1, 0):
        ops = _ops(api, ls, s, kind, "f64", target_cb)
        O = _oracle_op(oracle, s, kind, target_cb)
        ins = [lat.spinor().upload(sl.cut_spinor(psi)) for sl, lat in zip(ls.slabs, ls.lats)]
        outs = [lat.spinor() for lat in ls.lats]
        for isign in (1, -1):
            ls.eo_apply(ops, outs, ins, isign, target_cb)
            got = np.concatenate([o.download() for o in outs])
            assert rel_l2(got, O.apply(psi, isign, target_cb)) < 1e-13, (kind, nslabs, target_cb, isign)


def test_one_slab_equals_the_one_gpu_operator(api, setup):
    """With one slab the faces wrap onto the slab itself: the halo path must
    reproduce the one-GPU clover operator exactly."""
    s = setup
    ls = halo.LocalSlabs(DIMS, 1)
    ops = _ops(api, ls, s, "clover", "f64", 1)
    lat = ls.lats[0]
    psi = F.gaussian_spinor(DIMS, 8)
    x = lat.spinor().upload(psi)
    y = lat.spinor()
    ls.eo_apply(ops, [y], [x], 1, 1)
    u = lat.gauge("f64", 12).upload(s["gauge"])
    M = api.EvenOddCloverOperator(u, lat.clover().upload(s["clov"][1]), lat.clover().upload(s["invclov"][0]),
                                  -1.0, *ANISO)
    z = lat.spinor()
    M(z, x, 1, 1)
    assert rel_l2(y.download(), z.download()) < 1e-14


def test_halo_refuses_twisted_phases_and_two_flavours(api, setup):
    s = setup
    ls = halo.LocalSlabs(DIMS, 2)
    lat = ls.lats[0]
    u = lat.gauge("f64", 12).upload(ls.slabs[0].cut_gauge(s["gauge"]))
    x, y = lat.spinor("f64", 2), lat.spinor("f64", 2)
    buf = __import__("torch").zeros(1 << 20, dtype=__import__("torch").uint8, device="cuda:0")
    f = halo.faces_struct(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), ls.slabs[0])
    p = api.op_params(L.WILSON, -1.0, use_tbc=[0, 0, 0, 1], tbc_phases=[[1, 0]] * 3 + [[0.6, 0.8]])
    assert L._lib.qphix_gpu_dslash_halo(C.byref(p), y.h, x.h, u.h, None, None, 1, 0, C.byref(f)) != 0
    p = api.op_params(L.NDTM, mass=0.1, twisted_mass=0.2, epsilon=0.1)
    assert L._lib.qphix_gpu_dslash_halo(C.byref(p), y.h, x.h, u.h, None, None, 1, 0, C.byref(f)) != 0


def test_slab_operator_with_exchange_faces_one_slab(api, setup):
    """The per-rank path (SlabOperator with exchange_faces) on one slab: the
    exchange returns the slab's own faces, so the operator must equal the
    one-GPU clover operator."""
    s = setup
    slab = halo.TSlab(DIMS, 1, 0)
    lat = api.Lattice(slab.dims)
    u = lat.gauge("f64", 12).upload(s["gauge"])
    A = lat.clover().upload(s["clov"][1])
    Ai = lat.clover().upload(s["invclov"][0])
    p = api.op_params(L.CLOVER_OP, -1.0, *ANISO)
    M = halo.SlabOperator(slab, lat, p, u, lambda f, l: halo.exchange_faces(f, l, slab), clov=A, invclov=Ai)
    x = lat.spinor().upload(F.gaussian_spinor(DIMS, 9))
    y, z = lat.spinor(), lat.spinor()
    for isign in (1, -1):
        M(y, x, isign, 1)
        api.EvenOddCloverOperator(u, A, Ai, -1.0, *ANISO)(z, x, isign, 1)
        assert rel_l2(y.download(), z.download()) < 1e-14


@pytest.mark.parametrize("nslabs", [2, 4])
def test_slab_cg_matches_one_gpu_cg(api, oracle, setup, nslabs):
    """CG on M^+ M with the clover operator over 2 / 4 slabs (faces exchanged
    every application, norms summed over the slabs) converges like the one-GPU
    solver: the same iteration count (within one), the true residual below the
    target, and the solutions equal to 1e-8."""
    s = setup
    ls = halo.LocalSlabs(DIMS, nslabs)
    ops = _ops(api, ls, s, "clover", "f64", 1)
    b = F.gaussian_spinor(DIMS, 11)
    bs = [lat.spinor().upload(sl.cut_spinor(b)) for sl, lat in zip(ls.slabs, ls.lats)]
    xs = [lat.spinor() for lat in ls.lats]
    it, rr = halo.cg(lambda outs, ins, isign: ls.eo_apply(ops, outs, ins, isign, 1), xs, bs, 1e-10, 2000)
    x = np.concatenate([f.download() for f in xs])
    O = _oracle_op(oracle, s, "clover", 1)
    r = b - O.apply(O.apply(x, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10 and rr < 1e-20
    xo, io = oracle.cg(O, b, 1e-10, 2000)
    assert abs(it - io.n_iters) <= 1, (it, io.n_iters)
    assert rel_l2(x, xo) < 1e-8
