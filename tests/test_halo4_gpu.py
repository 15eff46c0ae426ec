"""Halo mode for a lattice cut along any of x, y, z, t (qphix_b200/halo.py
Block / LocalBlocks, qphix_gpu_dslash_halo4), emulated on one GPU: the
lattice is cut into a grid of blocks, each on its own lattice object, every
block packs the faces of each cut direction and reads its neighbours'
(LocalBlocks), and the glued result equals the whole-lattice oracle:
relative L2 <= 1e-13 in FP64 and the stated FP16 tolerance in FP16, for both
checkerboards and isign, with antiperiodic time and anisotropic hops; a CG
on M^+ M over a 2 x 2 x 2 x 2 grid reaches the oracle's solution."""
import numpy as np
import pytest

from helpers import TOL, make_setup, rel_l2
from qphix_b200 import _lib as L
from qphix_b200 import fields as F
from qphix_b200 import halo

pytestmark = pytest.mark.gpu
DIMS = (8, 4, 4, 8)
ANISO = (0.9, 1.1)
GRIDS = [(2, 1, 1, 1), (1, 2, 1, 1), (1, 1, 2, 1), (1, 1, 1, 2), (2, 2, 2, 2)]


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def setup():
    return make_setup(DIMS, seed=63, gauge_kind="weak", mass=0.1, mu=0.07)


def _ops(api, lb, s, kind, prec, target_cb):
    p = api.op_params({"wilson": L.WILSON, "clover": L.CLOVER_OP, "tm": L.TM, "tmclover": L.TMCLOVER}[kind],
                      -1.0, ANISO[0], ANISO[1], mass=s["mass"], twisted_mass=s["mu"],
                      prec_mass_rho=s["mu"] if kind == "tmclover" else 0.0)
    other = 1 - target_cb

    def make(block, lat, exchange):
        u = lat.gauge(prec, 12).upload(block.cut_gauge(s["gauge"]))
        kw = {}
        if kind == "clover":
            kw = dict(clov=lat.clover(prec).upload(block.cut_clover(s["clov"][target_cb])),
                      invclov=lat.clover(prec).upload(block.cut_clover(s["invclov"][other])))
        elif kind == "tmclover":
            f0, f1 = s["finv"][other]
            kw = dict(clov=lat.clover(prec).upload(block.cut_clover(s["clov"][target_cb])),
                      finv=(lat.full_clover(prec).upload(block.cut_clover(f0)),
                            lat.full_clover(prec).upload(block.cut_clover(f1))))
        return halo.BlockOperator(block, lat, p, u, exchange, **kw)
    return lb.operators(make)


def _glue(lb, outs, like):
    whole = np.zeros_like(like)
    for b, o in zip(lb.blocks, outs):
        b.glue_spinor(whole, o.download())
    return whole


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


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("prec", ["f64", "f16"])
def test_halo4_wilson_dslash(api, oracle, setup, grid, prec):
    s = setup
    lb = halo.LocalBlocks(DIMS, grid)
    ops = _ops(api, lb, s, "wilson", prec, 1)
    Lg = oracle.make_lattice(DIMS, -1.0, *ANISO)
    psi = np.stack([F.gaussian_spinor(DIMS, 9), F.gaussian_spinor(DIMS, 10)])
    ins = [lat.spinor(prec, 2).upload(b.cut_spinor(psi)) for b, lat in zip(lb.blocks, lb.lats)]
    outs = [lat.spinor(prec, 2) for lat in lb.lats]
    for isign in (1, -1):
        for cb in (0, 1):
            lb.dslash(ops, outs, ins, isign, cb)
            got = _glue(lb, outs, psi)
            for k in range(2):
                ref = oracle.dslash(Lg, psi[k], s["gauge"], isign, cb)
                assert rel_l2(got[k], ref) < TOL[prec], (grid, prec, isign, cb, k)


@pytest.mark.parametrize("kind", ["wilson", "clover", "tm", "tmclover"])
@pytest.mark.parametrize("grid", [(2, 1, 2, 1), (2, 2, 2, 2)])
def test_halo4_eo_operators(api, oracle, setup, kind, grid):
    s = setup
    lb = halo.LocalBlocks(DIMS, grid)
    psi = F.gaussian_spinor(DIMS, 11)
    for target_cb in (1, 0):
        ops = _ops(api, lb, s, kind, "f64", target_cb)
        O = _oracle_op(oracle, s, kind, target_cb)
        ins = [lat.spinor().upload(b.cut_spinor(psi)) for b, lat in zip(lb.blocks, lb.lats)]
        outs = [lat.spinor() for lat in lb.lats]
        for isign in (1, -1):
            lb.eo_apply(ops, outs, ins, isign, target_cb)
            got = _glue(lb, outs, psi)
            assert rel_l2(got, O.apply(psi, isign, target_cb)) < 1e-13, (kind, grid, target_cb, isign)


def test_halo4_t_cut_equals_the_slab_path(api, setup):
    """A t-only grid through qphix_gpu_dslash_halo4 gives the same numbers as
    the t-slab entry point qphix_gpu_dslash_halo."""
    s = setup
    lb = halo.LocalBlocks(DIMS, (1, 1, 1, 2))
    ls = halo.LocalSlabs(DIMS, 2)
    ops4 = _ops(api, lb, s, "clover", "f64", 1)
    p = ops4[0].p

    def make(slab, lat, exchange):
        u = lat.gauge("f64", 12).upload(slab.cut_gauge(s["gauge"]))
        return halo.SlabOperator(slab, lat, p, u, exchange,
                                 clov=lat.clover().upload(slab.cut_clover(s["clov"][1])),
                                 invclov=lat.clover().upload(slab.cut_clover(s["invclov"][0])))
    ops1 = ls.operators(make)
    psi = F.gaussian_spinor(DIMS, 12)
    a = [lat.spinor() for lat in lb.lats]
    b = [lat.spinor() for lat in ls.lats]
    lb.eo_apply(ops4, a, [lat.spinor().upload(bl.cut_spinor(psi)) for bl, lat in zip(lb.blocks, lb.lats)], 1, 1)
    ls.eo_apply(ops1, b, [lat.spinor().upload(sl.cut_spinor(psi)) for sl, lat in zip(ls.slabs, ls.lats)], 1, 1)
    for x, y in zip(a, b):
        assert np.array_equal(x.download(), y.download())


def test_halo4_cg(api, oracle, setup):
    """CG on M^+ M (halo.cg) over a 2 x 2 x 2 x 2 grid of blocks reaches the
    oracle's CG solution."""
    s = setup
    lb = halo.LocalBlocks(DIMS, (2, 2, 2, 2))
    ops = _ops(api, lb, s, "clover", "f64", 1)
    b = F.gaussian_spinor(DIMS, 13)
    gb = [lat.spinor().upload(bl.cut_spinor(b)) for bl, lat in zip(lb.blocks, lb.lats)]
    gx = [lat.spinor() for lat in lb.lats]
    it, rr = halo.cg(lambda outs, ins, isign: lb.eo_apply(ops, outs, ins, isign, 1), gx, gb, 1e-10, 2000)
    x = _glue(lb, gx, b)
    O = _oracle_op(oracle, s, "clover", 1)
    r = b - O.apply(O.apply(x, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    xo, io = oracle.cg(O, b, 1e-10, 2000)
    assert abs(it - io.n_iters) <= 1
    assert rel_l2(x, xo) < 1e-8


def test_halo4_refuses_bad_cuts(api, setup):
    import ctypes as C

    import torch
    s = setup
    lb = halo.LocalBlocks(DIMS, (2, 1, 1, 1))
    lat = lb.lats[0]
    u = lat.gauge("f64", 12).upload(lb.blocks[0].cut_gauge(s["gauge"]))
    x, y = lat.spinor(), lat.spinor()
    buf = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda:0")
    p = api.op_params(L.WILSON, -1.0)
    f = halo.faces4_struct(lb.blocks[0], {0: buf.data_ptr()}, {0: buf.data_ptr()}, {0: buf.data_ptr()})
    f.cut = 0  # no cut direction
    assert L._lib.qphix_gpu_dslash_halo4(C.byref(p), y.h, x.h, u.h, None, None, 1, 0, C.byref(f)) != 0
    f.cut = 1 | 2  # y cut without its face buffers
    assert L._lib.qphix_gpu_dslash_halo4(C.byref(p), y.h, x.h, u.h, None, None, 1, 0, C.byref(f)) != 0
