"""Even-odd operators and solvers through the C ABI against the CPU oracle.

Operators: relative L2 <= 1e-13 (FP64) / 1e-6 (FP32) for every kind, isign
and target checkerboard, plus the gamma_5 hermiticity identity
|<y, M x> - <M^dag y, x>| / (|y| |M x|) <= 1e-14 in FP64
(the idea of include/qphix/inv_dummy_hermtest.h).
Solvers: the true residual |b - M x| / |b| is recomputed in FP64 for every
solve and must meet the target; FP64 iteration counts equal the oracle's
(same recurrences as include/qphix/invcg.h, invbicgstab.h, invmr.h).
"""
import numpy as np
import pytest

from helpers import TOL, make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu

KINDS = ["wilson", "clover", "tm", "tmclover"]


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def setup():
    return make_setup((4, 4, 4, 8), seed=21, gauge_kind="weak", mass=0.1, mu=0.1)


def build_ops(api, oracle, s, kind, prec="f64", recon=12, target_cb=1):
    dims = s["dims"]
    lat = api.Lattice(dims)
    u = lat.gauge(prec, recon).upload(s["gauge"])
    L = oracle.make_lattice(dims, -1.0, 1.0, 1.0)
    other = 1 - target_cb
    keep = [u]
    if kind == "wilson":
        M = api.EvenOddWilsonOperator(s["mass"], u)
        O = oracle.OracleOp("wilson", L, s["gauge"], mass=s["mass"])
    elif kind == "tm":
        M = api.EvenOddTMWilsonOperator(s["mass"], s["mu"], u)
        O = oracle.OracleOp("tm", L, s["gauge"], mass=s["mass"], twisted_mass=s["mu"])
    elif kind == "clover":
        A = lat.clover(prec).upload(s["clov"][target_cb])
        Ai = lat.clover(prec).upload(s["invclov"][other])
        keep += [A, Ai]
        M = api.EvenOddCloverOperator(u, A, Ai, prec_mass_rho=0.0)
        O = oracle.OracleOp("clover", L, s["gauge"], clov=s["clov"][target_cb],
                            invclov=s["invclov"][other])
    else:
        A = lat.clover(prec).upload(s["clov"][target_cb])
        f0 = lat.full_clover(prec).upload(s["finv"][other][0])
        f1 = lat.full_clover(prec).upload(s["finv"][other][1])
        keep += [A, f0, f1]
        M = api.EvenOddTMCloverOperator(u, A, (f0, f1), prec_mass_rho=s["mu"])
        O = oracle.OracleOp("tmclover", L, s["gauge"], clov=s["clov"][target_cb],
                            finv=s["finv"][other], rho=s["mu"])
    M._keep = keep
    return lat, M, O


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_eo_operator(api, oracle, setup, kind, prec):
    for target_cb in (1, 0):
        lat, M, O = build_ops(api, oracle, setup, kind, prec, target_cb=target_cb)
        x = F.gaussian_spinor(setup["dims"], 31)
        gx = lat.spinor(prec).upload(x)
        gr = lat.spinor(prec)
        for isign in (1, -1):
            M(gr, gx, isign, target_cb)
            ref = O.apply(x, isign, target_cb)
            assert rel_l2(gr.download(), ref) < TOL[prec], (kind, target_cb, isign)


@pytest.mark.parametrize("kind", KINDS)
def test_hermiticity(api, oracle, setup, kind):
    lat, M, O = build_ops(api, oracle, setup, kind)
    x = F.gaussian_spinor(setup["dims"], 32)
    y = F.gaussian_spinor(setup["dims"], 33)
    gx, gy = lat.spinor().upload(x), lat.spinor().upload(y)
    mx, mdy = lat.spinor(), lat.spinor()
    M(mx, gx, 1)
    M(mdy, gy, -1)
    a = np.vdot(y, mx.download())
    b = np.vdot(mdy.download(), x)
    assert abs(a - b) / (np.linalg.norm(y) * np.linalg.norm(mx.download())) < 1e-14


@pytest.mark.parametrize("kind", KINDS)
def test_cg(api, oracle, setup, kind):
    lat, M, O = build_ops(api, oracle, setup, kind)
    b = F.gaussian_spinor(setup["dims"], 41)
    gx, gb = lat.spinor(), lat.spinor().upload(b)
    info = api.InvCG(M, 500)(gx, gb, 1e-10)[0]
    xo, io = oracle.cg(O, b, 1e-10, 500)
    x = gx.download()
    r = b - O.apply(O.apply(x, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10 * 1.5
    assert info["status"] == 0 and info["true_rel_resid"] < 1.5e-10
    assert info["n_iters"] == io.n_iters
    assert rel_l2(x, xo) < 1e-8


@pytest.mark.parametrize("kind", KINDS)
def test_bicgstab(api, oracle, setup, kind):
    lat, M, O = build_ops(api, oracle, setup, kind)
    b = F.gaussian_spinor(setup["dims"], 42)
    gx, gb = lat.spinor(), lat.spinor().upload(b)
    info = api.InvBiCGStab(M, 500)(gx, gb, 1e-10)[0]
    xo, io = oracle.bicgstab(O, b, 1e-10, 500)
    x = gx.download()
    r = b - O.apply(x, 1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10
    assert info["status"] == 0
    assert abs(info["n_iters"] - io.n_iters) <= 1
    assert rel_l2(x, xo) < 1e-8


@pytest.mark.parametrize("omega", [1.0, 1.1, 0.8])
def test_mr(api, oracle, setup, omega):
    """InvMR (invmr.h:62-210) with over-relaxation: iteration count and
    solution equal the oracle's for Omega != 1 too."""
    lat, M, O = build_ops(api, oracle, setup, "clover")
    b = F.gaussian_spinor(setup["dims"], 43)
    gx, gb = lat.spinor(), lat.spinor().upload(b)
    info = api.InvMR(M, 2000, omega)(gx, gb, 1e-10)[0]
    xo, io = oracle.mr(O, b, 1e-10, 2000, omega)
    x = gx.download()
    r = b - O.apply(x, 1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10
    assert info["n_iters"] == io.n_iters
    assert rel_l2(x, xo) < 1e-9


@pytest.mark.parametrize("omega", [1.0, 1.2])
def test_mr_smoother(api, oracle, setup, omega):
    """InvMRSmoother (invmr.h:294-354): exactly n MR iterations, no residual
    test, rsd_sq_final = -1; the same iterates as the oracle's MR run to an
    unreachable target for n iterations."""
    lat, M, O = build_ops(api, oracle, setup, "tmclover")
    b = F.gaussian_spinor(setup["dims"], 44)
    for n in (1, 7):
        gx, gb = lat.spinor(), lat.spinor().upload(b)
        info = api.InvMRSmoother(M, n, omega)(gx, gb)[0]
        xo, io = oracle.mr(O, b, 0.0, n, omega)
        assert io.n_iters == n and info["n_iters"] == n
        assert info["rsd_sq_final"] == -1
        assert rel_l2(gx.download(), xo) < 1e-12, n


@pytest.mark.parametrize("inner_prec", ["f32", "f16", "bf16", "q16"])
def test_richardson_mixed(api, oracle, setup, inner_prec):
    s = setup
    lat, M, O = build_ops(api, oracle, s, "clover")
    u_in = lat.gauge(inner_prec, 12).upload(s["gauge"])
    A = lat.clover(inner_prec).upload(s["clov"][1])
    Ai = lat.clover(inner_prec).upload(s["invclov"][0])
    Mi = api.EvenOddCloverOperator(u_in, A, Ai)
    b = F.gaussian_spinor(s["dims"], 44)
    gx, gb = lat.spinor(), lat.spinor().upload(b)
    solver = api.InvRichardsonMultiPrec(M, Mi, "bicgstab", delta=0.1, max_iters=50)
    info = solver(gx, gb, 1e-10)[0]
    x = gx.download()
    r = b - O.apply(x, 1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    assert info["status"] == 0


def test_multi_rhs_block_matches_single(api, oracle, setup):
    """A block of right-hand sides gives, rhs by rhs, the single-rhs result."""
    s = setup
    dims = s["dims"]
    for prec in ("f64", "f32"):
        lat, M, O = build_ops(api, oracle, s, "clover", prec)
        nr = 4
        bs = [F.gaussian_spinor(dims, 50 + i) for i in range(nr)]
        gb = lat.spinor(prec, nr).upload(np.stack(bs))
        gr = lat.spinor(prec, nr)
        M(gr, gb, 1)
        out = gr.download()
        for i in range(nr):
            assert rel_l2(out[i], O.apply(bs[i], 1)) < TOL[prec]
        gx = lat.spinor(prec, nr)
        infos = api.InvBiCGStab(M, 500)(gx, gb, 1e-5 if prec == "f32" else 1e-10)
        xs = gx.download()
        for i in range(nr):
            r = bs[i] - O.apply(xs[i], 1)
            assert np.linalg.norm(r) / np.linalg.norm(bs[i]) < (2e-5 if prec == "f32" else 2e-10)
            assert infos[i]["status"] == 0


@pytest.mark.parametrize("kind", ["wilson", "clover"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_minvcg(api, oracle, setup, kind, prec):
    """Multishift CG (include/qphix/minvcg.h): same iteration count as the
    oracle in FP64, every shifted system solved to its target."""
    lat, M, O = build_ops(api, oracle, setup, kind, prec)
    b = F.gaussian_spinor(setup["dims"], 61)
    shifts = [1e-4, 1e-3, 0.01, 0.1, 1.0]
    tol = 1e-9 if prec == "f64" else 1e-5
    gb = lat.spinor(prec).upload(b)
    xs = [lat.spinor(prec) for _ in shifts]
    it, fin, mv = api.MInvCG(M, 2000)(xs, gb, shifts, [tol] * len(shifts))
    xo, io, fo, mvo = oracle.minvcg(O, b, shifts, [tol] * len(shifts), 2000)
    if prec == "f64":
        assert it == io and mv == mvo
    for s, x in zip(shifts, xs):
        xv = x.download()
        r = b - (O.apply(O.apply(xv, 1), -1) + s * xv)
        assert np.linalg.norm(r) / np.linalg.norm(b) < (3 * tol if prec == "f64" else 50 * tol), s
    if prec == "f64":
        for x, xr in zip(xs, xo):
            assert rel_l2(x.download(), xr) < 1e-7


@pytest.mark.parametrize("low", ["f16", "bf16", "q16", "q16f32", "f32"])
@pytest.mark.parametrize("nrhs", [1, 3])
def test_bicgstab_reliable_update(api, oracle, setup, low, nrhs):
    """BiCGStab with reliable updates (FP64 true residuals, low-precision
    iterations): every right-hand side reaches 1e-10 in the FP64 true
    residual, recomputed here with the oracle."""
    s = setup
    lat, M, O = build_ops(api, oracle, s, "clover")
    u_l = lat.gauge(low, 12).upload(s["gauge"])
    A = lat.clover(low).upload(s["clov"][1])
    Ai = lat.clover(low).upload(s["invclov"][0])
    Ml = api.EvenOddCloverOperator(u_l, A, Ai)
    bs = [F.gaussian_spinor(s["dims"], 80 + i) for i in range(nrhs)]
    gb = lat.spinor("f64", nrhs).upload(np.stack(bs))
    gx = lat.spinor("f64", nrhs)
    infos = api.InvBiCGStabMixed(M, Ml, delta=0.1)(gx, gb, 1e-10)
    xs = gx.download()
    if nrhs == 1:
        xs = xs[None]
    for i in range(nrhs):
        r = bs[i] - O.apply(xs[i], 1)
        assert np.linalg.norm(r) / np.linalg.norm(bs[i]) < 1e-10
        assert infos[i]["status"] == 0 and infos[i]["true_rel_resid"] < 1e-10


def _low_op(api, lat, s, kind, low, target_cb=1):
    other = 1 - target_cb
    u = lat.gauge(low, 12).upload(s["gauge"])
    keep = [u]
    if kind == "wilson":
        M = api.EvenOddWilsonOperator(s["mass"], u)
    elif kind == "tm":
        M = api.EvenOddTMWilsonOperator(s["mass"], s["mu"], u)
    elif kind == "clover":
        A = lat.clover(low).upload(s["clov"][target_cb])
        Ai = lat.clover(low).upload(s["invclov"][other])
        keep += [A, Ai]
        M = api.EvenOddCloverOperator(u, A, Ai)
    else:
        A = lat.clover(low).upload(s["clov"][target_cb])
        f0 = lat.full_clover(low).upload(s["finv"][other][0])
        f1 = lat.full_clover(low).upload(s["finv"][other][1])
        keep += [A, f0, f1]
        M = api.EvenOddTMCloverOperator(u, A, (f0, f1), prec_mass_rho=s["mu"])
    M._keep = keep
    return M


@pytest.mark.parametrize("kind", ["wilson", "tm", "tmclover"])
@pytest.mark.parametrize("low", ["f16", "bf16", "q16", "q16f32"])
def test_bicgstab_reliable_update_kinds(api, oracle, setup, kind, low):
    """The batched mixed solve for every operator kind (two right-hand sides,
    16-bit inner iterations): each reaches 1e-10 in the FP64 true residual,
    recomputed with the oracle's operator."""
    s = setup
    lat, M, O = build_ops(api, oracle, s, kind)
    Ml = _low_op(api, lat, s, kind, low)
    bs = [F.gaussian_spinor(s["dims"], 90 + i) for i in range(2)]
    gb = lat.spinor("f64", 2).upload(np.stack(bs))
    gx = lat.spinor("f64", 2)
    infos = api.InvBiCGStabMixed(M, Ml, delta=0.1)(gx, gb, 1e-10)
    xs = gx.download()
    for i in range(2):
        r = bs[i] - O.apply(xs[i], 1)
        assert np.linalg.norm(r) / np.linalg.norm(bs[i]) < 1e-10, (kind, low, i)
        assert infos[i]["status"] == 0


def test_multishift_fp32_with_fp64_refinement(api, oracle, setup):
    """FP32 multishift CG on M^+M followed by FP64 defect correction of each
    shift (FP64 residual, FP32 single-shift corrections): every shift's
    solution meets 1e-9 in the FP64 true residual of (M^+M + shift),
    recomputed with the oracle."""
    s = setup
    lat, M64, O = build_ops(api, oracle, s, "wilson")
    M32 = _low_op(api, lat, s, "wilson", "f32")
    shifts = [1e-3, 1e-2, 0.1, 1.0]
    tol = 1e-9
    b = F.gaussian_spinor(s["dims"], 123)
    b64, b32 = lat.spinor("f64").upload(b), lat.spinor("f32").upload(b)
    xs32 = [lat.spinor("f32") for _ in shifts]
    api.MInvCG(M32, 2000)(xs32, b32, shifts, [tol] * len(shifts))
    r64, t64, o64, d64 = (lat.spinor("f64") for _ in range(4))
    r32, d32 = lat.spinor("f32"), lat.spinor("f32")
    one = api.MInvCG(M32, 2000, max_shifts=1)
    bn = np.linalg.norm(b)
    for k, sh in enumerate(shifts):
        x64 = lat.spinor("f64")
        x64.convert_from(xs32[k])
        for _ in range(10):
            M64(t64, x64, 1)
            M64(o64, t64, -1)
            api.caxpby(sh, x64, 1.0, o64)
            api.copy(r64, b64)
            api.caxpby(-1.0, o64, 1.0, r64)
            rn = float(np.sqrt(api.norm2(r64)[0]))
            if rn / bn < tol:
                break
            r32.convert_from(r64, 1.0 / rn)
            api.zero(d32)
            one([d32], r32, [sh], [max(1e-5, 0.3 * tol * bn / rn)])
            d64.convert_from(d32, rn)
            api.caxpby(1.0, d64, 1.0, x64)
        x = x64.download()
        r = b - (O.apply(O.apply(x, 1), -1) + sh * x)
        assert np.linalg.norm(r) / bn < tol, (sh, np.linalg.norm(r) / bn)


@pytest.mark.parametrize("kind", KINDS)
def test_cg_shifted(api, oracle, setup, kind):
    """CG on (M^+M + s_i) x_i = b_i, one shift per right-hand side
    (qphix_gpu_solve_cg_shifted): every system meets its target by the
    oracle's true residual, and takes the oracle's shifted CG's iteration
    count (within one: |r|^2 and |p|^2 are summed in BLAS passes, in another
    order than the oracle's) to the same solution."""
    lat, M, O = build_ops(api, oracle, setup, kind)
    shifts = [0.0, 1e-3, 0.05, 1.0]
    tol = 1e-10
    bs = [F.gaussian_spinor(setup["dims"], 140 + i) for i in range(len(shifts))]
    gb = lat.spinor("f64", len(shifts)).upload(np.stack(bs))
    gx = lat.spinor("f64", len(shifts))
    api.zero(gx)
    infos = api.InvCGShifted(M, 2000)(gx, gb, shifts, tol)
    xs = gx.download()
    for i, sh in enumerate(shifts):
        r = bs[i] - (O.apply(O.apply(xs[i], 1), -1) + sh * xs[i])
        rel = np.linalg.norm(r) / np.linalg.norm(bs[i])
        assert rel < tol, (kind, sh, rel)
        assert infos[i]["status"] == 0
        assert abs(infos[i]["true_rel_resid"] - rel) <= 1e-3 * rel + 1e-16
    for i, sh in enumerate(shifts):
        xo, io = oracle.cg_shift(O, bs[i], sh, tol, 2000)
        assert abs(infos[i]["n_iters"] - io.n_iters) <= 1, (kind, sh, infos[i]["n_iters"], io.n_iters)
        assert rel_l2(xs[i], xo) < 1e-8, (kind, sh)
    # larger shifts converge in fewer iterations
    assert infos[3]["n_iters"] < infos[1]["n_iters"]


@pytest.mark.parametrize("kind", ["wilson", "clover"])
@pytest.mark.parametrize("low,rsd_low", [("f32", None), ("f16", 1e-3)])
def test_mshift_mixed(api, oracle, setup, kind, low, rsd_low):
    """Multishift CG in low precision plus the batched refinement of every
    shift (qphix_gpu_solve_mshift_cg_mixed): each shift meets 1e-9 by the
    oracle's FP64 true residual of (M^+M + shift), and the solutions agree
    with the FP64 multishift CG's."""
    s = setup
    lat, M64, O = build_ops(api, oracle, s, kind)
    Ml = _low_op(api, lat, s, kind, low)
    shifts = [1e-4, 1e-3, 0.01, 0.1, 1.0]
    tol = 1e-9
    b = F.gaussian_spinor(s["dims"], 151)
    gb = lat.spinor("f64").upload(b)
    xs = [lat.spinor("f64") for _ in shifts]
    out = api.MInvCGMixed(M64, Ml, 5000)(xs, gb, shifts, [tol] * len(shifts), rsd_low=rsd_low)
    assert out["corrections"] >= 1 and out["refine_iters"] > 0
    bn = np.linalg.norm(b)
    for k, sh in enumerate(shifts):
        x = xs[k].download()
        r = b - (O.apply(O.apply(x, 1), -1) + sh * x)
        rel = np.linalg.norm(r) / bn
        assert rel < tol, (kind, low, sh, rel)
        assert abs(out["true_rel_resid"][k] - rel) <= 1e-3 * rel + 1e-16
    ref = [lat.spinor("f64") for _ in shifts]
    api.MInvCG(M64, 5000)(ref, gb, shifts, [tol] * len(shifts))
    for x, xr in zip(xs, ref):
        assert rel_l2(x.download(), xr.download()) < 1e-7


def test_mshift_mixed_zero_source(api, oracle, setup):
    """A zero source gives zero solutions without iterating."""
    s = setup
    lat, M64, O = build_ops(api, oracle, s, "wilson")
    Ml = _low_op(api, lat, s, "wilson", "f32")
    gb = lat.spinor("f64")
    api.zero(gb)
    xs = [lat.spinor("f64").upload(F.gaussian_spinor(s["dims"], 160 + k)) for k in range(3)]
    out = api.MInvCGMixed(M64, Ml, 100)(xs, gb, [1e-3, 0.1, 1.0], [1e-9] * 3)
    assert out["n_iters"] == 0 and out["corrections"] == 0 and out["mv_apps"] == 0
    for x in xs:
        assert not np.any(x.download())


def test_fused_blas_entry_points():
    """qphix_gpu_blas_caxpby_norm2 / _xmy_norm2 / _inner_product_norm
    (axpyNorm2, xmyNorm2Spinor, innerProductNorm of include/qphix/blas_new_c.h)
    against numpy, FP64, two right-hand sides."""
    from qphix_b200 import api
    dims = (4, 4, 4, 8)
    lat = api.Lattice(dims)
    xs = np.stack([F.gaussian_spinor(dims, 300 + k) for k in range(2)])
    ys = np.stack([F.gaussian_spinor(dims, 310 + k) for k in range(2)])
    x = lat.spinor("f64", 2).upload(xs)
    y = lat.spinor("f64", 2).upload(ys)
    ip, nx = api.inner_product_norm(x, y)
    for k in range(2):
        assert abs(ip[k] - np.vdot(xs[k], ys[k])) < 1e-12 * abs(ip[k])
        assert abs(nx[k] - np.vdot(xs[k], xs[k]).real) < 1e-12 * nx[k]
    z = lat.spinor("f64", 2)
    n = api.xmy_norm2(x, y, z)
    assert np.allclose(z.download(), xs - ys, rtol=0, atol=1e-14)
    assert np.allclose(n, [np.vdot(xs[k] - ys[k], xs[k] - ys[k]).real for k in range(2)], rtol=1e-12)
    n = api.caxpby_norm2(0.5 - 0.25j, x, 2.0, y)
    ref = (0.5 - 0.25j) * xs + 2.0 * ys
    assert np.allclose(y.download(), ref, rtol=0, atol=1e-14)
    assert np.allclose(n, [np.vdot(ref[k], ref[k]).real for k in range(2)], rtol=1e-12)
