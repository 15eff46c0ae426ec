"""Parity at the benchmarked configurations and launch shapes (GPU).

The headline (16^3x32 clover, kappa 0.1360, links exp(i 0.3 H), 8 rhs), the
batched twisted-mass clover configuration (24^3x48, 24 rhs, BF16 storage) and
the multishift configuration (16 log-spaced shifts) run here in the shapes
the bench launches, and every result is checked by something the library
did not compute:
  - operator outputs against the CPU oracle (itself pinned to QPhiX's own
    kernels): 1e-13 (FP64), 1e-6 (FP32), 4e-3 (FP16), 3e-2 (BF16) relative L2;
  - the reductions fused into the A chi - b D psi epilogue (|res|^2, <w, res>,
    <res, chi>), which at 16^3x32 fold 256-512 site blocks per rhs, against
    numpy on the downloaded fields: 1e-12 (FP64), 1e-6 (FP32); 16-bit
    storage rounds the stored output after the sums are taken, so there the
    bound is the storage error, 3e-3;
  - the headline solver's solutions by the oracle's FP64 operator:
    |b - M x| / |b| <= 1e-10 for every rhs;
  - multishift iteration count and solutions against the oracle's
    multishift CG (include/qphix/minvcg.h:279-384).
"""
import os
import sys

import numpy as np
import pytest

from helpers import TOL, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
C2 = (16, 16, 16, 32)
NORM_TOL = {"f64": 1e-12, "f32": 1e-6, "f16": 3e-3}


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def c2():
    sys.path.insert(0, ROOT)
    import bench
    return bench.make_inputs(C2, 8)


@pytest.fixture(scope="module")
def c2_oracle(oracle, c2):
    L = oracle.make_lattice(C2, -1.0)
    return L, oracle.OracleOp("clover", L, c2["gauge"], clov=c2["clov_odd"], invclov=c2["invclov_even"])


SHAPE_ENV = {"sp1": {"QPHIX_GPU_RHS_TILE": "1", "QPHIX_GPU_SITES_PER_THREAD": "1"},
             "r2": {"QPHIX_GPU_RHS_TILE": "2", "QPHIX_GPU_SITES_PER_THREAD": "1"},
             "sp2": {"QPHIX_GPU_RHS_TILE": "1", "QPHIX_GPU_SITES_PER_THREAD": "2"},
             "rhs_lanes": {"QPHIX_GPU_RHS_LANES": "1"}}


class forced_shape:
    """Force the Dslash launch shape (rhs per thread, sites per thread, or two
    rhs in the float2 lanes) through the library's QPHIX_GPU_RHS_TILE /
    QPHIX_GPU_SITES_PER_THREAD / QPHIX_GPU_RHS_LANES."""

    def __init__(self, name):
        self.env = SHAPE_ENV[name]

    def __enter__(self):
        os.environ.update(self.env)

    def __exit__(self, *exc):
        for k in self.env:
            os.environ.pop(k, None)


def test_c2_fp64_operator_8rhs(api, c2, c2_oracle):
    L, O = c2_oracle
    lat = api.Lattice(C2)
    u = lat.gauge("f64", 12).upload(c2["gauge"])
    A = lat.clover("f64").upload(c2["clov_odd"])
    Ai = lat.clover("f64").upload(c2["invclov_even"])
    M = api.EvenOddCloverOperator(u, A, Ai)
    x = lat.spinor("f64", 8).upload(c2["rhs"])
    y = lat.spinor("f64", 8)
    for isign in (1, -1):
        M(y, x, isign, 1)
        got = y.download()
        for r in range(8):
            assert rel_l2(got[r], O.apply(c2["rhs"][r], isign, 1)) < 1e-13, (isign, r)


@pytest.mark.parametrize("prec", ["f16", "f32", "f64"])
@pytest.mark.parametrize("shape", ["sp1", "r2", "sp2", "rhs_lanes"])
def test_c2_inner_kernels_every_shape(api, oracle, c2, c2_oracle, prec, shape):
    """The inner operator's two clover Dslash launches at 16^3x32 x 8 rhs in
    each built launch shape: A^-1 D psi and A chi - b D psi with the three
    fused reductions, against the oracle and numpy."""
    L, _ = c2_oracle
    lat = api.Lattice(C2)
    u = lat.gauge(prec, 12).upload(c2["gauge"])
    A = lat.clover(prec).upload(c2["clov_odd"])
    Ai = lat.clover(prec).upload(c2["invclov_even"])
    rhs = c2["rhs"]
    chi_h = np.stack([F.gaussian_spinor(C2, 500 + r) for r in range(8)])
    w_h = np.stack([F.gaussian_spinor(C2, 600 + r) for r in range(8)])
    psi = lat.spinor(prec, 8).upload(rhs)
    chi = lat.spinor(prec, 8).upload(chi_h)
    w = lat.spinor(prec, 8).upload(w_h)
    tmp = lat.spinor(prec, 8)
    out = lat.spinor(prec, 8)
    D = api.ClovDslash(lat, -1.0, 1.0, 1.0)
    with forced_shape(shape):
        D.dslash(tmp, psi, u, Ai, 1, 0)
        norms = D.dslashAChiMinusBDPsiNorms(out, tmp, chi, u, A, 0.25, 1, 1, w=w)
    tol = TOL[prec]
    t_gpu = tmp.download()
    o_gpu = out.download()
    # stored (rounded) inputs, as the kernels read them
    psi_s, chi_s, w_s = psi.download(), chi.download(), w.download()
    for r in range(8):
        t_ref = oracle.clov_dslash(L, psi_s[r], c2["gauge"], c2["invclov_even"], 1, 0)
        assert rel_l2(t_gpu[r], t_ref) < tol, ("dslash", r)
        o_ref = oracle.clov_achimbdpsi(L, t_gpu[r], chi_s[r], c2["gauge"], c2["clov_odd"], 0.25, 0.0, 1, 1)
        assert rel_l2(o_gpu[r], o_ref) < tol, ("achimbdpsi", r)
        n2 = np.vdot(o_gpu[r], o_gpu[r]).real
        wo = np.vdot(w_s[r], o_gpu[r])
        oc = np.vdot(o_gpu[r], chi_s[r])
        scale = np.sqrt(n2) * np.sqrt(np.vdot(chi_s[r], chi_s[r]).real)
        nt = NORM_TOL[prec]
        assert abs(norms[r, 0] - n2) <= nt * n2, ("|res|^2", r)
        assert abs(complex(norms[r, 1], norms[r, 2]) - wo) <= nt * scale, ("<w,res>", r)
        assert abs(complex(norms[r, 3], norms[r, 4]) - oc) <= nt * scale, ("<res,chi>", r)


def test_c2_headline_solutions_checked_by_oracle(api, c2, c2_oracle):
    """The headline solve (InvRichardsonMultiPrec, FP64 outer, FP16-storage
    BiCGStab inner, delta 0.005, 8 rhs) reaches 1e-10 by the oracle's FP64
    operator, not only by the library's own residual."""
    L, O = c2_oracle
    lat = api.Lattice(C2)
    u64 = lat.gauge("f64", 12).upload(c2["gauge"])
    M64 = api.EvenOddCloverOperator(u64, lat.clover("f64").upload(c2["clov_odd"]),
                                    lat.clover("f64").upload(c2["invclov_even"]))
    ui = lat.gauge("f16", 12).upload(c2["gauge"])
    Mi = api.EvenOddCloverOperator(ui, lat.clover("f16").upload(c2["clov_odd"]),
                                   lat.clover("f16").upload(c2["invclov_even"]))
    solver = api.InvRichardsonMultiPrec(M64, Mi, "bicgstab", delta=0.005, max_iters=100, inner_max_iters=5000)
    b = lat.spinor("f64", 8).upload(c2["rhs"])
    x = lat.spinor("f64", 8)
    api.zero(x)
    infos = solver(x, b, 1e-10)
    xs = x.download()
    for r in range(8):
        assert infos[r]["status"] == 0
        res = c2["rhs"][r] - O.apply(xs[r], 1, 1)
        rel = np.linalg.norm(res) / np.linalg.norm(c2["rhs"][r])
        assert rel <= 1.01e-10, (r, rel)
        assert abs(rel - infos[r]["true_rel_resid"]) <= 1e-3 * rel, r


def _c3_fields(api, dims):
    """The batched twisted-mass clover configuration's fields, built on the
    device as the benchmark builds them (qphix_b200.workloads.c3)."""
    kappa, mu, csw = 0.1373, 0.01, 1.0
    mass = F.kappa_to_mass(kappa)
    g = F.make_gauge(dims, 301, "exp", eps=0.4)
    lat = api.Lattice(dims)
    u64 = lat.gauge("f64", 12).upload(g)
    a_odd = api.clover_build(lat.clover("f64"), u64, 1, mass, csw)
    a_even = api.clover_build(lat.clover("f64"), u64, 0, mass, csw)
    f0, f1 = lat.full_clover("f64"), lat.full_clover("f64")
    api.clover_invert_twisted(f0, f1, a_even, mu)
    srcs = [F.point_source(dims, s, c) for s in range(4) for c in range(3)]
    srcs += [F.z2_noise(dims, 400 + i) for i in range(12)]
    return lat, g, u64, a_odd, (f0, f1), np.stack(srcs), mu


def test_c3_tmclover_24rhs_bf16_and_fp64(api, oracle):
    """24^3x48 twisted-mass clover even-odd operator on the 24-rhs block
    (12 point + 12 Z2 sources): BF16 storage / FP32 arithmetic and FP64,
    against the oracle on right-hand sides spread over the block (both
    halves, first and last)."""
    dims = (24, 24, 24, 48)
    lat, g, u64, a_odd, finv, srcs, mu = _c3_fields(api, dims)
    A_h = a_odd.download().reshape(-1, 2, 36)
    f_h = [f.download().reshape(-1, 2, 6, 6, 2) for f in finv]
    f_h = [f[..., 0] + 1j * f[..., 1] for f in f_h]
    L = oracle.make_lattice(dims, -1.0)
    O = oracle.OracleOp("tmclover", L, g, clov=A_h, finv=f_h, rho=mu)
    ulo = lat.gauge("bf16", 12).upload(g)
    a_lo = api.clover_convert(lat.clover("bf16"), a_odd)
    f_lo = (api.clover_convert(lat.full_clover("bf16"), finv[0]),
            api.clover_convert(lat.full_clover("bf16"), finv[1]))
    check = [0, 7, 11, 12, 18, 23]
    for prec, M, tol in (("f64", api.EvenOddTMCloverOperator(u64, a_odd, finv, prec_mass_rho=mu), 1e-13),
                         ("bf16", api.EvenOddTMCloverOperator(ulo, a_lo, f_lo, prec_mass_rho=mu), TOL["bf16"])):
        x = lat.spinor(prec, 24).upload(srcs)
        y = lat.spinor(prec, 24)
        M(y, x, 1, 1)
        got = y.download()
        xin = x.download()
        for r in check:
            ref = O.apply(xin[r], 1, 1)
            assert rel_l2(got[r], ref) < tol, (prec, r)


def test_c4_multishift_16_shifts(api, oracle):
    """Multishift CG on Wilson M^+ M with the 16 log-spaced shifts of the
    multishift configuration (kappa 0.125, tolerance 1e-9), on 8^3x16: FP64
    iteration count equal to the oracle's, every shift's solution against
    the oracle's and its true residual by the oracle's operator."""
    dims = (8, 8, 8, 16)
    mass = F.kappa_to_mass(0.125)
    g = F.make_gauge(dims, 41, "exp", eps=0.3)
    shifts = list(np.logspace(-4, 0, 16))
    tol = 1e-9
    b = F.gaussian_spinor(dims, 42)
    lat = api.Lattice(dims)
    u = lat.gauge("f64", 12).upload(g)
    M = api.EvenOddWilsonOperator(mass, u)
    L = oracle.make_lattice(dims, -1.0)
    O = oracle.OracleOp("wilson", L, g, mass=mass)
    gb = lat.spinor("f64").upload(b)
    xs = [lat.spinor("f64") for _ in shifts]
    it, fin, mv = api.MInvCG(M, 5000)(xs, gb, shifts, [tol] * len(shifts))
    xo, io, fo, mvo = oracle.minvcg(O, b, shifts, [tol] * len(shifts), 5000)
    assert it == io and mv == mvo
    for s, x, xr in zip(shifts, xs, xo):
        xv = x.download()
        r = b - (O.apply(O.apply(xv, 1), -1) + s * xv)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 3 * tol, s
        assert rel_l2(xv, xr) < 1e-7, s
