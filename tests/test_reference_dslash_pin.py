"""Pins the CPU oracle's Dslash family, its even-odd operators and the
QPhiX-layout packer of qphix_b200.fields to QPhiX's own code-generated
kernels (CPU only).

The reference side is QPhiX itself: its code generator's kernels
(codegen/dslash_common.cc) behind its Dslash / ClovDslash / TMDslash /
TMClovDslash classes and EvenOdd*Operator templates, built from the reference
sources by oracle/ref/codegen.mk into oracle/_ref/libqphix_ref_dslash_*.so
(scalar: veclen = soalen = 1; avx512: double veclen 8 with soalen 4 / 8,
float veclen 16 with soalen 8).  Inputs are random SU(3) links (not unit
links, so U, U^T and U^+ differ), packed by QPhiXLayout into the blocked
layout the reference reads, and the result is unpacked the same way; a wrong
transposition, back-link placement or 12-real compression in the packer, or
a wrong sign, projector or boundary factor in the oracle, shows up as a
mismatch.  Tolerances: 1e-13 relative L2 in double, 1e-6 in float
(reference float kernels against the double oracle).

Where the reference library is absent, the oracle is checked against
tests/golden/reference_dslash_pin.npz (projections of the reference outputs on
seeded vectors, written by tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from helpers import make_setup, rel_l2
from qphix_b200 import fields as F

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "reference_dslash_pin.npz")
DIMS = (8, 4, 4, 8)       # Nx/2 = 4: scalar and the avx512 double soalen-4 layout
DIMS_WIDE = (16, 4, 4, 4)  # Nx/2 = 8: avx512 soalen 8 (double veclen 8, float veclen 16)
KINDS = ["wilson", "clover", "tm", "tmclover"]
OPS = {"wilson": ["dslash", "achimbdpsi", "eo"], "clover": ["dslash", "achimbdpsi", "clovmult", "eo"],
       "tm": ["dslash", "achimbdpsi", "eo"], "tmclover": ["dslash", "achimbdpsi", "eo"]}
MASS, MU, RHO = 0.1, 0.07, 0.03
ALPHA, BETA = 1.3, 0.27


def _R():
    import ref_dslash as R  # test infrastructure: QPhiX's own kernels
    return R


def _need(isa):
    R = _R()
    if not R.available(isa):
        pytest.skip(f"reference {isa} Dslash library not built or not runnable on this host")
    return R


def setup_fields(dims, seed=5):
    s = make_setup(dims, seed=seed, gauge_kind="gaussian", mass=MASS, mu=MU)
    return s, F.gaussian_spinor(dims, seed + 1), F.gaussian_spinor(dims, seed + 2)


def case(R, RL, O, s, kind, op, isign, cb, t_bc, aniso, psi, chi, gp):
    """(reference output, oracle output) of one call."""
    dims = s["dims"]
    a_s, a_t = aniso
    L = O.make_lattice(dims, t_bc, a_s, a_t)
    p = R.params(t_boundary=t_bc, aniso_s=a_s, aniso_t=a_t, mass=MASS, mu=MU, alpha=ALPHA, beta=BETA)
    g = s["gauge"]
    other = 1 - cb
    if op == "eo":
        if kind == "wilson":
            c, oo = (None, None, None), O.OracleOp("wilson", L, g, mass=MASS)
        elif kind == "tm":
            c, oo = (None, None, None), O.OracleOp("tm", L, g, mass=MASS, twisted_mass=MU)
        elif kind == "clover":
            p[5] = RHO
            c = (RL.clover(s["clov"][cb]), RL.clover(s["invclov"][other]), None)
            oo = O.OracleOp("clover", L, g, clov=s["clov"][cb], invclov=s["invclov"][other], rho=RHO)
        else:
            p[5] = MU
            c = (RL.clover(s["clov"][cb]), RL.full_clover(s["finv"][other][0]),
                 RL.full_clover(s["finv"][other][1]))
            oo = O.OracleOp("tmclover", L, g, clov=s["clov"][cb], finv=s["finv"][other], rho=MU)
        return RL.apply(kind, "eo", psi, gp, isign, cb, c=c, p=p), oo.apply(psi, isign, cb)
    if kind == "wilson":
        if op == "dslash":
            return RL.apply(kind, op, psi, gp, isign, cb, p=p), O.dslash(L, psi, g, isign, cb)
        return (RL.apply(kind, op, psi, gp, isign, cb, chi=chi, p=p),
                O.dslash_achimbdpsi(L, psi, chi, g, ALPHA, BETA, isign, cb))
    if kind == "clover":
        p[5] = RHO
        if op == "dslash":
            return (RL.apply(kind, op, psi, gp, isign, cb, c=(RL.clover(s["invclov"][cb]), None, None), p=p),
                    O.clov_dslash(L, psi, g, s["invclov"][cb], isign, cb))
        if op == "clovmult":
            return (RL.apply(kind, op, psi, gp, isign, cb, c=(RL.clover(s["clov"][cb]), None, None), p=p),
                    O.clover_apply(psi, s["clov"][cb]))
        return (RL.apply(kind, op, psi, gp, isign, cb, chi=chi, c=(RL.clover(s["clov"][cb]), None, None), p=p),
                O.clov_achimbdpsi(L, psi, chi, g, s["clov"][cb], BETA, RHO, isign, cb))
    if kind == "tm":
        if op == "dslash":
            return RL.apply(kind, op, psi, gp, isign, cb, p=p), O.tm_dslash(L, psi, g, MASS, MU, isign, cb)
        musign = -1.0 if isign < 0 else 1.0
        p[8] = musign
        return (RL.apply(kind, op, psi, gp, isign, cb, chi=chi, p=p),
                O.tm_achimbdpsi(L, psi, chi, g, ALPHA, BETA, MASS, MU, isign, cb, musign))
    p[5] = MU
    if op == "dslash":
        f = s["finv"][cb]
        return (RL.apply(kind, op, psi, gp, isign, cb, c=(RL.full_clover(f[0]), RL.full_clover(f[1]), None), p=p),
                O.tmclov_dslash(L, psi, g, f[0], f[1], isign, cb))
    return (RL.apply(kind, op, psi, gp, isign, cb, chi=chi, c=(RL.clover(s["clov"][cb]), None, None), p=p),
            O.clov_achimbdpsi(L, psi, chi, g, s["clov"][cb], BETA, MU, isign, cb))


@pytest.fixture(scope="module")
def fields():
    return setup_fields(DIMS)


@pytest.mark.parametrize("compress12", [False, True])
@pytest.mark.parametrize("kind", KINDS)
def test_scalar_reference_matches_oracle(oracle, fields, kind, compress12):
    R = _need("scalar")
    s, psi, chi = fields
    RL = R.RefLattice(DIMS, "double", "scalar", compress12=compress12, nthreads=4)
    gp = RL.gauge(s["gauge"])
    for op in OPS[kind]:
        for isign in (1, -1):
            for cb in (0, 1):
                for t_bc, aniso in ((-1.0, (1.0, 1.0)), (1.0, (0.9, 1.2))):
                    ref, orc = case(R, RL, oracle, s, kind, op, isign, cb, t_bc, aniso, psi, chi, gp)
                    assert rel_l2(ref, orc) < 1e-13, (op, isign, cb, t_bc)


@pytest.mark.parametrize("compress12", [False, True])
def test_scalar_reference_dslash_dir(oracle, fields, compress12):
    """Dslash::dslashDir (dslash_body.h:350-358): one hop direction at a time."""
    R = _need("scalar")
    s, psi, _ = fields
    RL = R.RefLattice(DIMS, "double", "scalar", compress12=compress12, nthreads=4)
    gp = RL.gauge(s["gauge"])
    L = oracle.make_lattice(DIMS, -1.0, 0.9, 1.2)
    for d in range(8):
        for cb in (0, 1):
            ref = RL.apply("wilson", "dir", psi, gp, 1, cb, p=R.params(t_boundary=-1.0, aniso_s=0.9, aniso_t=1.2, dir=d))
            assert rel_l2(ref, oracle.dslash_dir(L, psi, s["gauge"], cb, d)) < 1e-13, (d, cb)


@pytest.mark.parametrize("kind", KINDS)
def test_scalar_reference_float_kernels(oracle, fields, kind):
    """The reference's float kernels against the double oracle: 1e-6."""
    R = _need("scalar")
    s, psi, chi = fields
    RL = R.RefLattice(DIMS, "float", "scalar", compress12=True, nthreads=4)
    gp = RL.gauge(s["gauge"])
    for op in OPS[kind]:
        for isign in (1, -1):
            ref, orc = case(R, RL, oracle, s, kind, op, isign, 1, -1.0, (1.0, 1.0), psi, chi, gp)
            assert rel_l2(ref, orc) < 1e-6, (op, isign)


@pytest.mark.parametrize("compress12", [False, True])
@pytest.mark.parametrize("kind", KINDS)
def test_avx512_reference_blocked_layout(oracle, fields, kind, compress12):
    """veclen 8 / soalen 4 (two y rows per vector): the blocked layout with
    nGY = 2 that the scalar build does not exercise."""
    R = _need("avx512")
    s, psi, chi = fields
    RL = R.RefLattice(DIMS, "double", "avx512", veclen=8, soalen=4, compress12=compress12, nthreads=4)
    gp = RL.gauge(s["gauge"])
    for op in OPS[kind]:
        for isign in (1, -1):
            for cb in (0, 1):
                ref, orc = case(R, RL, oracle, s, kind, op, isign, cb, -1.0, (1.0, 1.0), psi, chi, gp)
                assert rel_l2(ref, orc) < 1e-13, (op, isign, cb)


@pytest.mark.parametrize("prec,veclen,tol", [("double", 8, 1e-13), ("float", 16, 1e-6)])
def test_avx512_reference_soalen8(oracle, prec, veclen, tol):
    R = _need("avx512")
    s, psi, chi = setup_fields(DIMS_WIDE, seed=9)
    RL = R.RefLattice(DIMS_WIDE, prec, "avx512", veclen=veclen, soalen=8, compress12=True, nthreads=4)
    gp = RL.gauge(s["gauge"])
    for kind in KINDS:
        for op in OPS[kind]:
            ref, orc = case(R, RL, oracle, s, kind, op, 1, 1, -1.0, (1.0, 1.0), psi, chi, gp)
            assert rel_l2(ref, orc) < tol, (kind, op)


@pytest.mark.parametrize("veclen,soalen,compress12", [(1, 1, False), (4, 2, True), (8, 4, False), (16, 8, True)])
def test_gauge_pack_round_trip(veclen, soalen, compress12):
    """QPhiXLayout.pack_gauge / unpack_gauge / unpack_back_gauge invert each
    other: forward links U_mu(x) in the odd slots, U_mu(x - mu) of the other
    checkerboard in the even slots (qdp_packer_parscalar.h:94-129)."""
    dims = (16, 4, 4, 4)
    g = F.make_gauge(dims, 3, "gaussian")
    lay = F.QPhiXLayout(dims, veclen, soalen, compress12)
    for cb in (0, 1):
        blk = lay.pack_gauge(g, cb)
        assert np.abs(lay.unpack_gauge(blk) - g[cb]).max() < 1e-14
        back = lay.unpack_back_gauge(blk)
        x = F.cb_coords(dims, cb)
        for mu in range(4):
            c = list(x)
            c[mu] = (c[mu] - 1) % dims[mu]
            sb = ((c[3] * dims[2] + c[2]) * dims[1] + c[1]) * (dims[0] // 2) + c[0] // 2
            assert np.abs(back[mu] - g[1 - cb, mu, sb]).max() < 1e-14


def _golden_inputs():
    s, psi, chi = setup_fields(DIMS)
    rng = np.random.default_rng(77)
    probes = F.gaussian_complex(rng, (3, F.vh(DIMS), 4, 3))
    return s, psi, chi, probes


def golden_cases():
    """(name, kind, op, isign, cb, compress12) of the golden fixture"""
    out = []
    for kind in KINDS:
        for op in OPS[kind]:
            for isign in (1, -1):
                for cb in (0, 1):
                    out.append((f"{kind}_{op}_{isign:+d}_{cb}", kind, op, isign, cb))
    return out


def project(v, probes):
    """norm and inner products with the probe vectors: a size-independent
    fingerprint of one output"""
    return np.concatenate([[np.vdot(v, v).real], [np.vdot(p, v) for p in probes]])


def test_oracle_against_golden_reference_outputs(oracle):
    """The committed fingerprints of the reference's outputs (scalar build,
    18-real links, antiperiodic t) against the oracle, wherever the
    reference is absent or present."""
    if not os.path.exists(GOLD):
        pytest.skip("golden fixture not generated")
    gold = dict(np.load(GOLD))
    s, psi, chi, probes = _golden_inputs()

    class OracleOnly:  # the oracle half of case() only
        @staticmethod
        def params(**kw):
            return np.zeros(10)

    class NoRef:
        def clover(self, c):
            return None

        def full_clover(self, c):
            return None

        def gauge(self, g):
            return None

        def apply(self, *a, **k):
            return np.zeros((F.vh(DIMS), 4, 3), complex)

    for name, kind, op, isign, cb in golden_cases():
        _, orc = case(OracleOnly, NoRef(), oracle, s, kind, op, isign, cb, -1.0, (1.0, 1.0), psi, chi, None)
        fp = project(orc, probes)
        ref = gold[name]
        assert np.abs(fp - ref).max() <= 1e-12 * abs(ref[0]), name
