"""The C++ drop-in headers (include/qphix/) used the way a QPhiX caller uses
QPhiX: tests/cpp/dropin_main.cc is compiled with g++ against the headers and
the library, fed QPhiX-layout host arrays (Geometry<double,4,2,true> with
padding, and Geometry<float,8,2,true> for the inner solver of
InvRichardsonMultiPrec) packed from seeded fields, and its outputs -- a
Dslash, the clover operator, BiCGStab, CG, Richardson and multishift-CG
solves, the two-flavour twisted-mass Wilson and clover operators and their
CG solves, the ClovDslash members, InvMR / InvMRSmoother with over-relaxation,
and the twisted-mass Wilson and twisted-mass clover operators -- are
checked against the CPU oracle.  An UnprecSolverWrapper solve of the full
(unpreconditioned) clover system is checked through its full residual."""
import os
import subprocess

import numpy as np
import pytest

from helpers import make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_dropin(tmp_path, oracle):
    exe = tmp_path / "dropin"
    subprocess.check_call(["g++", "-std=c++14", "-O1", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "dropin_main.cc"),
                           "-L", os.path.join(ROOT, "qphix_b200"), "-lqphix_b200",
                           "-Wl,-rpath," + os.path.join(ROOT, "qphix_b200"), "-o", str(exe)])
    dims = (8, 4, 4, 8)
    s = make_setup(dims, seed=31, gauge_kind="weak", mass=0.1)
    d = tmp_path
    np.array(dims, dtype=np.int32).tofile(d / "dims")
    np.array([s["mass"]], dtype=np.float64).tofile(d / "mass")
    # Geometry(latt, By=2, Bz=2, 1, 1, 1, PadXY=1, PadXYZ=1): double V=4 S=2 / float V=8 S=2
    for tag, V, S, dt in (("d_", 4, 2, np.float64), ("f_", 8, 2, np.float32)):
        lay = F.QPhiXLayout(dims, V, S, True, pad_xy=1, pad_xyz=1)
        for cb in range(2):
            lay.pack_gauge(s["gauge"], cb, dt).tofile(d / f"{tag}u{cb}")
        lay.pack_clover(s["clov"][1], dt).tofile(d / f"{tag}A_odd")
        lay.pack_clover(s["invclov"][0], dt).tofile(d / f"{tag}Ainv_even")
    lay = F.QPhiXLayout(dims, 4, 2, True, pad_xy=1, pad_xyz=1)
    psi = F.gaussian_spinor(dims, 32)
    lay.pack_spinor(psi)[1:].tofile(d / "d_psi")  # block 0 = what allocCBFourSpinor returns
    chi = F.gaussian_spinor(dims, 33)
    lay.pack_spinor(chi)[1:].tofile(d / "d_chi")
    nd = (s["mass"], 0.3, 0.2)  # mass, mu, epsilon of the two-flavour operators
    np.array(nd, dtype=np.float64).tofile(d / "ndtm")
    ndc_fu, ndc_fd, ndc_c = F.ndtm_clover_inverses(s["clov"][0], nd[1], nd[2])
    lay.pack_clover(ndc_c).tofile(d / "d_ndc_odiag")
    lay.pack_full_clover(ndc_fu).tofile(d / "d_ndc_fup")
    lay.pack_full_clover(ndc_fd).tofile(d / "d_ndc_fdn")
    g2 = F.make_gauge(dims, 77, "weak")  # a second gauge field for the cache checks
    lay.pack_gauge(g2, 0).tofile(d / "d_u0b")
    mu_tm = 0.07
    np.array([mu_tm], dtype=np.float64).tofile(d / "tm_mu")
    tinv = F.twisted_full_inverse(s["clov"][0], mu_tm)
    lay.pack_full_clover(tinv[0]).tofile(d / "d_tm_finv0")
    lay.pack_full_clover(tinv[1]).tofile(d / "d_tm_finv1")
    out = subprocess.run([str(exe), str(d)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr + out.stdout

    def load(name):
        a = np.fromfile(d / name, dtype=np.float64)
        full = np.zeros((lay.n_spinor_blocks,) + (3, 4, 2, 2))
        full[1:] = a.reshape((-1, 3, 4, 2, 2))
        return lay.unpack_spinor(full)

    L = oracle.make_lattice(dims, -1.0)
    assert rel_l2(load("out_dslash"), oracle.dslash(L, psi, s["gauge"], 1, 0)) < 1e-13
    O = oracle.OracleOp("clover", L, s["gauge"], clov=s["clov"][1], invclov=s["invclov"][0])
    assert rel_l2(load("out_clover_op"), O.apply(psi, 1, 1)) < 1e-13
    x = load("out_bicgstab_x")
    assert np.linalg.norm(psi - O.apply(x, 1)) / np.linalg.norm(psi) < 2e-10
    info = np.fromfile(d / "out_bicgstab_info")
    xo, io = oracle.bicgstab(O, psi, 1e-10, 2000)
    assert abs(int(info[0]) - io.n_iters) <= 1
    W = oracle.OracleOp("wilson", L, s["gauge"], mass=s["mass"])
    y = load("out_cg_x")
    assert np.linalg.norm(psi - W.apply(W.apply(y, 1), -1)) / np.linalg.norm(psi) < 2e-10
    z = load("out_rich_x")
    assert np.linalg.norm(psi - O.apply(z, 1)) / np.linalg.norm(psi) < 1e-10
    for i, sh in enumerate((0.01, 0.1, 0.5)):
        xs = load(f"out_minv_x{i}")
        r = psi - (O.apply(O.apply(xs, 1), -1) + sh * xs)
        assert np.linalg.norm(r) / np.linalg.norm(psi) < 3e-9
    N = oracle.OracleOp("ndtm", L, s["gauge"], mass=nd[0], twisted_mass=nd[1], epsilon=nd[2])
    pair = np.stack([psi, chi])
    got = np.stack([load("out_nd_up"), load("out_nd_dn")])
    assert rel_l2(got, N.apply(pair, 1, 1)) < 1e-13
    xn = np.stack([load("out_ndcg_up"), load("out_ndcg_dn")])
    r = pair - N.apply(N.apply(xn, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(pair) < 2e-10
    NC = oracle.OracleOp("ndtmclover", L, s["gauge"], clov=s["clov"][1], invclov=ndc_c, finv=(ndc_fu, ndc_fd),
                         twisted_mass=nd[1], epsilon=nd[2])
    got = np.stack([load("out_ndc_up"), load("out_ndc_dn")])
    assert rel_l2(got, NC.apply(pair, 1, 1)) < 1e-13
    xn = np.stack([load("out_ndccg_up"), load("out_ndccg_dn")])
    r = pair - NC.apply(NC.apply(xn, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(pair) < 2e-10
    # Dslash-level two-flavour members (tm_clov_dslash_def.h:76-110, tm_dslash_def.h)
    got = np.stack([load("out_2f_inv_up"), load("out_2f_inv_dn")])
    ref = np.stack([oracle.fullclover_apply(psi, ndc_fu) + oracle.clover_apply(chi, ndc_c),
                    oracle.fullclover_apply(chi, ndc_fd) + oracle.clover_apply(psi, ndc_c)])
    assert rel_l2(got, ref) < 1e-13
    got = np.stack([load("out_2f_clachi_up"), load("out_2f_clachi_dn")])
    ref = np.stack([oracle.clov_achimbdpsi(L, psi, chi, s["gauge"], s["clov"][1], 0.25, nd[1], 1, 1) - nd[2] * psi,
                    oracle.clov_achimbdpsi(L, chi, psi, s["gauge"], s["clov"][1], 0.25, -nd[1], 1, 1) - nd[2] * chi])
    assert rel_l2(got, ref) < 1e-13
    got = np.stack([load("out_2f_tmachi_up"), load("out_2f_tmachi_dn")])
    al = 4.0 + nd[0]
    ref = np.stack([oracle.tm_achimbdpsi(L, psi, chi, s["gauge"], al, 0.25, nd[0], nd[1], -1, 1, 1.0) - nd[2] * psi,
                    oracle.tm_achimbdpsi(L, chi, psi, s["gauge"], al, 0.25, nd[0], nd[1], -1, 1, -1.0) - nd[2] * chi])
    assert rel_l2(got, ref) < 1e-13
    # BLAS of blas_new_c.h on host arrays
    sc = np.fromfile(d / "out_blas_scalars")
    assert abs(sc[0] - np.vdot(psi, psi).real) < 1e-12 * sc[0]
    ip = np.vdot(psi, chi)
    assert abs(sc[1] + 1j * sc[2] - ip) < 1e-12 * abs(ip) and abs(sc[3] + 1j * sc[4] - ip) < 1e-12 * abs(ip)
    assert abs(sc[5] - np.vdot(psi, psi).real) < 1e-12 * sc[5]
    assert abs(sc[6] - np.vdot(psi - chi, psi - chi).real) < 1e-12 * sc[6]
    c2 = (0.3 - 0.7j) * psi + chi + psi
    assert abs(sc[7] - np.vdot(c2, c2).real) < 1e-12 * sc[7] and sc[8] == 0.0
    for name, ref in (("axpy", psi + 0.5 * chi), ("axpby", 2 * psi - 1.5 * chi), ("xmy", psi - chi),
                      ("aypx", psi - 0.25 * chi), ("caxpy", (0.3 - 0.7j) * psi + chi), ("ax", 3 * (psi - chi))):
        assert rel_l2(load("out_blas_" + name), ref) < 1e-15, name
    assert rel_l2(load("out_blas_convert"), 2 * psi) < 1e-7  # through FP32
    # unpreconditioned clover system: [[A_ee, -D_eo/2], [-D_oe/2, A_oo]] x = (chi, psi)
    xe, xo = load("out_unprec_e"), load("out_unprec_o")
    re = oracle.clover_apply(xe, s["clov"][0]) - 0.5 * oracle.dslash(L, xo, s["gauge"], 1, 0) - chi
    ro = oracle.clover_apply(xo, s["clov"][1]) - 0.5 * oracle.dslash(L, xe, s["gauge"], 1, 1) - psi
    rel = np.sqrt((np.linalg.norm(re) ** 2 + np.linalg.norm(ro) ** 2)
                  / (np.linalg.norm(chi) ** 2 + np.linalg.norm(psi) ** 2))
    assert rel < 2e-10
    # ClovDslash members (clover_dslash_def.h:33-53), rho = 0.05
    assert rel_l2(load("out_clov_dslash"), oracle.clov_dslash(L, psi, s["gauge"], s["invclov"][0], 1, 0)) < 1e-13
    assert rel_l2(load("out_clov_achi"),
                  oracle.clov_achimbdpsi(L, psi, chi, s["gauge"], s["clov"][1], 0.25, 0.05, -1, 1)) < 1e-13
    assert rel_l2(load("out_clovmult"), oracle.clover_apply(psi, s["clov"][1])) < 1e-13
    # InvMR with Omega = 1.1 and InvMRSmoother (5 iterations, Omega = 1.2)
    xm, im = oracle.mr(O, psi, 1e-10, 2000, 1.1)
    info = np.fromfile(d / "out_mr_info")
    assert int(info[0]) == im.n_iters and rel_l2(load("out_mr_x"), xm) < 1e-9
    xs5, i5 = oracle.mr(O, psi, 0.0, 5, 1.2)
    info = np.fromfile(d / "out_mrs_info")
    assert int(info[0]) == 5 and info[1] == -1 and rel_l2(load("out_mrs_x"), xs5) < 1e-12
    # twisted-mass Wilson operator (twisted_mass.h:62-77) and BiCGStab on it;
    # twisted-mass clover operator (twisted_mass_clover.h:92-102), isign = -1
    TW = oracle.OracleOp("tm", L, s["gauge"], mass=s["mass"], twisted_mass=mu_tm)
    assert rel_l2(load("out_tmw_op"), TW.apply(psi, 1, 1)) < 1e-13
    xt = load("out_tmw_bicg_x")
    assert np.linalg.norm(psi - TW.apply(xt, 1)) / np.linalg.norm(psi) < 2e-10
    TC = oracle.OracleOp("tmclover", L, s["gauge"], clov=s["clov"][1], finv=tinv, rho=mu_tm)
    assert rel_l2(load("out_tmc_op"), TC.apply(psi, -1, 1)) < 1e-13
    # the cached device gauge copy: reused, invalidated after an in-place
    # rewrite, never matched for a reallocated array
    assert rel_l2(load("out_cache_1"), oracle.dslash(L, psi, s["gauge"], 1, 0)) < 1e-13
    assert rel_l2(load("out_cache_2"), oracle.dslash(L, psi, g2, 1, 0)) < 1e-13
    assert rel_l2(load("out_cache_3"), oracle.dslash(L, psi, g2, 1, 0)) < 1e-13
