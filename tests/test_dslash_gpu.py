"""Parity of the Dslash family through the C ABI against the CPU oracle.

Tolerances (relative L2 over the output checkerboard): FP64 1e-13, FP32 1e-6;
16-bit storage (FP32 arithmetic) is held to the stated bounds 4e-3 (FP16 +
per-site norm), 3e-2 (BF16 + per-site norm), 1e-3 (Q16: 16-bit fixed-point
spinors with per-site scale, FP16 links and clover) and 1e-4 (Q16F32: the same
spinors, FP32 links and clover) against the FP64 oracle.
Mirrors tests/testDslashFull.cc:110-168 (every isign, cb and t boundary).
"""
import numpy as np
import pytest

from helpers import TOL, make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu

DIMS = [(4, 4, 4, 8), (8, 4, 6, 4), (8, 8, 8, 8)]


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module", params=DIMS, ids=lambda d: "x".join(map(str, d)))
def setup(request):
    return make_setup(request.param)


def _fields(api, lat, s, prec, recon):
    u = lat.gauge(prec, recon).upload(s["gauge"])
    return u


@pytest.mark.parametrize("prec", ["f64", "f32", "f16", "bf16", "q16", "q16f32"])
@pytest.mark.parametrize("recon", [18, 12])
@pytest.mark.parametrize("t_bc", [1.0, -1.0])
def test_wilson_dslash(api, oracle, setup, prec, recon, t_bc):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, recon).upload(setup["gauge"])
    L = oracle.make_lattice(dims, t_bc, 0.35, 1.4)
    D = api.Dslash(lat, t_bc, 0.35, 1.4)
    psi = F.gaussian_spinor(dims, 5)
    chi = F.gaussian_spinor(dims, 6)
    gp = lat.spinor(prec).upload(psi)
    gc = lat.spinor(prec).upload(chi)
    gr = lat.spinor(prec)
    for isign in (1, -1):
        for cb in (0, 1):
            ref = oracle.dslash(L, psi, setup["gauge"], isign, cb)
            D.dslash(gr, gp, u, isign, cb)
            err = rel_l2(gr.download(), ref)
            assert err < TOL[prec], (prec, recon, isign, cb, err)
            ref = oracle.dslash_achimbdpsi(L, psi, chi, setup["gauge"], 0.7, 0.3, isign, cb)
            D.dslashAChiMinusBDPsi(gr, gp, gc, u, 0.7, 0.3, isign, cb)
            err = rel_l2(gr.download(), ref)
            assert err < TOL[prec], ("achimbdpsi", prec, recon, isign, cb, err)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_twisted_boundary_and_dir(api, oracle, setup, prec):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, 18).upload(setup["gauge"])
    ph = [np.exp(0.3j), np.exp(-0.7j), None, np.exp(1.1j)]
    use = [p is not None for p in ph]
    phases = [(p.real, p.imag) if p is not None else (1.0, 0.0) for p in ph]
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0, tbc=ph)
    D = api.Dslash(lat, -1.0, 1.0, 1.0, use, phases)
    psi = F.gaussian_spinor(dims, 7)
    gp = lat.spinor(prec).upload(psi)
    gr = lat.spinor(prec)
    for isign in (1, -1):
        ref = oracle.dslash(L, psi, setup["gauge"], isign, 0)
        D.dslash(gr, gp, u, isign, 0)
        assert rel_l2(gr.download(), ref) < TOL[prec]
    L0 = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    D0 = api.Dslash(lat, -1.0, 1.0, 1.0)
    for d in range(8):
        ref = oracle.dslash_dir(L0, psi, setup["gauge"], 1, d)
        D0.dslashDir(gr, gp, u, 1, d)
        assert rel_l2(gr.download(), ref) < TOL[prec], d


@pytest.mark.parametrize("prec", ["f64", "f32", "f16", "q16", "q16f32"])
@pytest.mark.parametrize("recon", [18, 12])
def test_clover_dslash(api, oracle, setup, prec, recon):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, recon).upload(setup["gauge"])
    rho = 0.17
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    D = api.ClovDslash(lat, -1.0, 1.0, 1.0, prec_mass_rho=rho)
    psi = F.gaussian_spinor(dims, 8)
    chi = F.gaussian_spinor(dims, 9)
    gp = lat.spinor(prec).upload(psi)
    gc = lat.spinor(prec).upload(chi)
    gr = lat.spinor(prec)
    for cb in (0, 1):
        A = lat.clover(prec).upload(setup["clov"][cb])
        Ai = lat.clover(prec).upload(setup["invclov"][cb])
        for isign in (1, -1):
            ref = oracle.clov_dslash(L, psi, setup["gauge"], setup["invclov"][cb], isign, cb)
            D.dslash(gr, gp, u, Ai, isign, cb)
            assert rel_l2(gr.download(), ref) < TOL[prec], ("dslash", cb, isign)
            ref = oracle.clov_achimbdpsi(L, psi, chi, setup["gauge"], setup["clov"][cb], 0.25, rho,
                                         isign, cb)
            D.dslashAChiMinusBDPsi(gr, gp, gc, u, A, 0.25, isign, cb)
            assert rel_l2(gr.download(), ref) < TOL[prec], ("achi", cb, isign)
        ref = oracle.clover_apply(chi, setup["clov"][cb])
        D.clovMult(gr, gc, A)
        assert rel_l2(gr.download(), ref) < TOL[prec], "clovMult"


@pytest.mark.parametrize("prec", ["f64", "f32", "f16"])
def test_tm_dslash(api, oracle, setup, prec):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, 12).upload(setup["gauge"])
    mass, mu = -0.2, 0.13
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    D = api.TMDslash(lat, -1.0, 1.0, 1.0, mass, mu)
    psi = F.gaussian_spinor(dims, 10)
    chi = F.gaussian_spinor(dims, 11)
    gp = lat.spinor(prec).upload(psi)
    gc = lat.spinor(prec).upload(chi)
    gr = lat.spinor(prec)
    for cb in (0, 1):
        for isign in (1, -1):
            ref = oracle.tm_dslash(L, psi, setup["gauge"], mass, mu, isign, cb)
            D.dslash(gr, gp, u, isign, cb)
            assert rel_l2(gr.download(), ref) < TOL[prec]
            for musign in (1.0, -1.0):
                ref = oracle.tm_achimbdpsi(L, psi, chi, setup["gauge"], 3.8, 0.25, mass, mu, isign, cb,
                                           musign)
                D.dslashAChiMinusBDPsi(gr, gp, gc, u, 3.8, 0.25, isign, cb, musign)
                assert rel_l2(gr.download(), ref) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32", "f16", "q16", "q16f32"])
def test_tmclover_dslash(api, oracle, setup, prec):
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, 12).upload(setup["gauge"])
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    D = api.TMClovDslash(lat, -1.0, 1.0, 1.0, prec_mass_rho=setup["mu"])
    psi = F.gaussian_spinor(dims, 12)
    gp = lat.spinor(prec).upload(psi)
    gr = lat.spinor(prec)
    for cb in (0, 1):
        f0, f1 = setup["finv"][cb]
        g0 = lat.full_clover(prec).upload(f0)
        g1 = lat.full_clover(prec).upload(f1)
        for isign in (1, -1):
            ref = oracle.tmclov_dslash(L, psi, setup["gauge"], f0, f1, isign, cb)
            D.dslash(gr, gp, u, (g0, g1), isign, cb)
            assert rel_l2(gr.download(), ref) < TOL[prec], (cb, isign)


def test_half_error_is_stated(api, oracle, setup):
    """16-bit storage: report the error against the FP64 oracle."""
    dims = setup["dims"]
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    psi = F.gaussian_spinor(dims, 13)
    ref = oracle.dslash(L, psi, setup["gauge"], 1, 0)
    errs = {}
    for prec in ("f32", "f16", "bf16", "q16", "q16f32"):
        lat = api.Lattice(dims)
        u = lat.gauge(prec, 12).upload(setup["gauge"])
        gp = lat.spinor(prec).upload(psi)
        gr = lat.spinor(prec)
        api.Dslash(lat, -1.0, 1.0, 1.0).dslash(gr, gp, u, 1, 0)
        errs[prec] = rel_l2(gr.download(), ref)
    print("relative L2 vs FP64 oracle:", errs)
    assert errs["f32"] < 1e-6 and errs["f16"] < 4e-3 and errs["bf16"] < 3e-2 and errs["q16"] < 1e-3 and errs["q16f32"] < 1e-4


SHAPES = [("sp1", {"QPHIX_GPU_SITES_PER_THREAD": "1", "QPHIX_GPU_RHS_TILE": "1"}),
          ("sp2", {"QPHIX_GPU_SITES_PER_THREAD": "2", "QPHIX_GPU_RHS_TILE": "1"}),
          ("r2", {"QPHIX_GPU_SITES_PER_THREAD": "1", "QPHIX_GPU_RHS_TILE": "2"}),
          ("rhs_lanes", {"QPHIX_GPU_RHS_LANES": "1"})]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: s[0])
@pytest.mark.parametrize("prec", ["f32", "f16", "bf16", "q16", "q16f32"])
@pytest.mark.parametrize("dims", [(6, 4, 4, 6), (8, 8, 8, 8)], ids=lambda d: "x".join(map(str, d)))
def test_launch_shapes(api, oracle, monkeypatch, shape, prec, dims):
    """Every built kernel shape (sites per thread, right-hand sides per
    thread, two right-hand sides in the float2 lanes) against the oracle with
    two right-hand sides, for every epilogue; 6x4x4x6 has 288 sites per
    checkerboard, so its last warp is only partly filled."""
    for k, v in shape[1].items():
        monkeypatch.setenv(k, v)
    s = make_setup(dims)
    lat = api.Lattice(dims)
    u = lat.gauge(prec, 12).upload(s["gauge"])
    u18 = lat.gauge(prec, 18).upload(s["gauge"])
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    psi = [F.gaussian_spinor(dims, 40 + i) for i in range(2)]
    chi = [F.gaussian_spinor(dims, 50 + i) for i in range(2)]
    gp = lat.spinor(prec, 2).upload(np.stack(psi))
    gc = lat.spinor(prec, 2).upload(np.stack(chi))
    gr = lat.spinor(prec, 2)
    D = api.Dslash(lat, -1.0, 1.0, 1.0)
    Cd = api.ClovDslash(lat, -1.0, 1.0, 1.0, prec_mass_rho=0.11)
    T = api.TMClovDslash(lat, -1.0, 1.0, 1.0, prec_mass_rho=s["mu"])
    Tm = api.TMDslash(lat, -1.0, 1.0, 1.0, s["mass"], s["mu"])
    for cb in (0, 1):
        A = lat.clover(prec).upload(s["clov"][cb])
        Ai = lat.clover(prec).upload(s["invclov"][cb])
        f0, f1 = s["finv"][cb]
        g0 = lat.full_clover(prec).upload(f0)
        g1 = lat.full_clover(prec).upload(f1)
        for isign in (1, -1):
            for links in (u, u18):
                D.dslash(gr, gp, links, isign, cb)
                out = gr.download()
                for i in range(2):
                    ref = oracle.dslash(L, psi[i], s["gauge"], isign, cb)
                    assert rel_l2(out[i], ref) < TOL[prec], ("wilson", cb, isign, i)
            Cd.dslash(gr, gp, u, Ai, isign, cb)
            out = gr.download()
            for i in range(2):
                ref = oracle.clov_dslash(L, psi[i], s["gauge"], s["invclov"][cb], isign, cb)
                assert rel_l2(out[i], ref) < TOL[prec], ("clover", cb, isign, i)
            Cd.dslashAChiMinusBDPsi(gr, gp, gc, u, A, 0.25, isign, cb)
            out = gr.download()
            for i in range(2):
                ref = oracle.clov_achimbdpsi(L, psi[i], chi[i], s["gauge"], s["clov"][cb], 0.25, 0.11, isign, cb)
                assert rel_l2(out[i], ref) < TOL[prec], ("achi", cb, isign, i)
            T.dslash(gr, gp, u, (g0, g1), isign, cb)
            out = gr.download()
            for i in range(2):
                ref = oracle.tmclov_dslash(L, psi[i], s["gauge"], f0, f1, isign, cb)
                assert rel_l2(out[i], ref) < TOL[prec], ("tmclover", cb, isign, i)
            D.dslashAChiMinusBDPsi(gr, gp, gc, u, 1.3, 0.27, isign, cb)
            out = gr.download()
            for i in range(2):
                ref = oracle.dslash_achimbdpsi(L, psi[i], chi[i], s["gauge"], 1.3, 0.27, isign, cb)
                assert rel_l2(out[i], ref) < TOL[prec], ("wilson achi", cb, isign, i)
            Tm.dslash(gr, gp, u, isign, cb)
            out = gr.download()
            for i in range(2):
                ref = oracle.tm_dslash(L, psi[i], s["gauge"], s["mass"], s["mu"], isign, cb)
                assert rel_l2(out[i], ref) < TOL[prec], ("tm", cb, isign, i)
            Tm.dslashAChiMinusBDPsi(gr, gp, gc, u, 4.0 + s["mass"], 0.25, isign, cb, -1.0)
            out = gr.download()
            for i in range(2):
                ref = oracle.tm_achimbdpsi(L, psi[i], chi[i], s["gauge"], 4.0 + s["mass"], 0.25, s["mass"], s["mu"],
                                           isign, cb, -1.0)
                assert rel_l2(out[i], ref) < TOL[prec], ("tm achi", cb, isign, i)


def test_autotuner_records_shapes(api, setup):
    """The tuner keeps one entry per Dslash configuration it has timed, with a
    built shape and a positive launch time."""
    dims = setup["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge("f16", 12).upload(setup["gauge"])
    gp = lat.spinor("f16", 2).upload(np.stack([F.gaussian_spinor(dims, 1), F.gaussian_spinor(dims, 2)]))
    gr = lat.spinor("f16", 2)
    api.Dslash(lat, -1.0, 1.0, 1.0).dslash(gr, gp, u, 1, 0)
    entries = api.tune_entries()
    key = "dslash p2 r12 e0 a0 %dx%dx%dx%d n2" % tuple(dims)
    assert key in entries, entries
    R, SP, us = entries[key]
    assert (R, SP) in [(1, 1), (1, 2), (2, 1), (2, 0)] and us > 0
