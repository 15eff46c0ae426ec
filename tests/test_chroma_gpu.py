"""QDP++ / Chroma CB2 host layout through the C ABI, and the Chroma-facing
LinOpSysSolver (qphix_b200/chroma.py) against the CPU oracle.

Layout: spinors (FP64 and FP32 arrays, one and two right-hand sides),
links and clover terms uploaded from CB2 full-lattice arrays equal the
canonical uploads bit for bit (FP64 arrays), and downloads write only the
requested checkerboard of the full array.

Solver: for each invType / SolverType, an anisotropic clover action given by
Kappa, with antiperiodic time, solves M psi_o = chi_o; the oracle operator
(built from the host clover term with the same coefficients) meets the
target on psi's odd checkerboard and psi's even checkerboard is untouched.
"""
import numpy as np
import pytest

from helpers import make_setup
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu
DIMS = (4, 4, 4, 8)


@pytest.fixture(scope="module")
def api():
    from qphix_b200 import api
    return api


@pytest.fixture(scope="module")
def setup():
    return make_setup(DIMS, seed=51, gauge_kind="weak", mass=0.1)


@pytest.mark.parametrize("dt", [np.complex128, np.complex64])
@pytest.mark.parametrize("nrhs", [1, 2])
def test_qdp_spinor_roundtrip(api, dt, nrhs):
    lat = api.Lattice(DIMS)
    vh = F.vh(DIMS)
    halves = [np.stack([F.gaussian_spinor(DIMS, 10 * cb + k) for k in range(nrhs)]) for cb in (0, 1)]
    full = F.qdp_spinor(*halves).astype(dt)
    if nrhs == 1:
        full = full[0]
    for cb in (0, 1):
        f = lat.spinor("f64", nrhs).upload_qdp(full, cb)
        got = f.download()
        want = F.qdp_spinor_cb(full, cb).astype(np.complex128)
        assert np.array_equal(got, want)
        out = np.full(full.shape, 7 + 7j, dtype=dt)
        f.download_qdp(out, cb)
        assert np.array_equal(F.qdp_spinor_cb(out, cb), F.qdp_spinor_cb(full, cb))
        assert np.all(F.qdp_spinor_cb(out, 1 - cb) == 7 + 7j)
        assert out.shape[-3] == 2 * vh


def test_qdp_gauge_and_clover_uploads(api, setup):
    s = setup
    lat = api.Lattice(DIMS)
    u_can = lat.gauge("f64", 12).upload(s["gauge"])
    u_qdp = lat.gauge("f64", 12).upload_qdp(F.qdp_gauge(s["gauge"]))
    D = api.Dslash(lat, -1.0, 1.0, 1.0)
    x = lat.spinor().upload(F.gaussian_spinor(DIMS, 3))
    a, b = lat.spinor(), lat.spinor()
    for cb in (0, 1):
        D.dslash(a, x, u_can, 1, cb)
        D.dslash(b, x, u_qdp, 1, cb)
        assert np.array_equal(a.download(), b.download())
    tri = F.qdp_clover(s["clov"])
    for cb in (0, 1):
        c_can = lat.clover().upload(s["clov"][cb])
        c_qdp = lat.clover().upload_qdp(tri, cb)
        assert np.array_equal(c_can.download(), c_qdp.download())
        out = np.full(tri.shape, -1.0)
        c_qdp.download_qdp(out, cb)
        vh = F.vh(DIMS)
        assert np.array_equal(out[cb * vh:(cb + 1) * vh], tri[cb * vh:(cb + 1) * vh])
        assert np.all(out[(1 - cb) * vh:(2 - cb) * vh] == -1.0)


XML = """<InvertParam>
  <invType>{inv}</invType>
  <SolverType>{solver}</SolverType>
  <MaxIter>{maxit}</MaxIter>
  <RsdTarget>1.0e-10</RsdTarget>
  <Delta>0.1</Delta>
  <CloverParams>
    <Kappa>0.118</Kappa>
    <clovCoeffR>1.3</clovCoeffR>
    <clovCoeffT>0.9</clovCoeffT>
    <AnisoParam><anisoP>true</anisoP><t_dir>3</t_dir><xi_0>1.6</xi_0><nu>1.1</nu></AnisoParam>
  </CloverParams>
  <AntiPeriodicT>true</AntiPeriodicT>
  <RsdToleranceFactor>{tolf}</RsdToleranceFactor>
  <Tune>false</Tune>
  <InnerType>{inner}</InnerType>
</InvertParam>"""


@pytest.mark.parametrize("inv,solver,inner,maxit", [
    ("QPHIX_CLOVER_INVERTER", "BICGSTAB", "h", 2000),
    ("QPHIX_CLOVER_INVERTER", "CG", "h", 4000),
    ("QPHIX_CLOVER_ITER_REFINE_BICGSTAB_INVERTER", "BICGSTAB", "f", 100),
    ("QPHIX_CLOVER_MIXED_BICGSTAB_INVERTER", "BICGSTAB", "h", 4000),
])
@pytest.mark.parametrize("nrhs", [1, 2])
def test_chroma_sys_solver(api, oracle, setup, inv, solver, inner, maxit, nrhs):
    from qphix_b200 import chroma
    s = setup
    # CG meets the target on the normal equations; M psi = chi is then looser
    tol = 1e-8 if solver == "CG" else 1e-9
    xml = XML.format(inv=inv, solver=solver, inner=inner, maxit=maxit, tolf=tol / 1e-10)
    solve = chroma.lin_op_sys_solver(xml, DIMS, F.qdp_gauge(s["gauge"]))
    cl = solve.param.clover
    chi = F.qdp_spinor(*[np.stack([F.gaussian_spinor(DIMS, 70 + 2 * k + cb) for k in range(nrhs)])
                         for cb in (0, 1)])
    if nrhs == 1:
        chi = chi[0]
    psi = np.zeros_like(chi)
    F.qdp_spinor_cb(psi, 0)[...] = 3.0
    res = solve(psi, chi)
    assert np.all(F.qdp_spinor_cb(psi, 0) == 3.0)
    # oracle: the same action from host-built clover terms
    dm, (cr, ct) = cl.diag_mass(), cl.clover_coeffs()
    A = F.make_clover(DIMS, s["gauge"], dm - 4.0, cr, ct)
    Ainv_e = F.invert_clover(A[0])
    as_, at = cl.aniso_factors()
    L = oracle.make_lattice(DIMS, -1.0, as_, at)
    O = oracle.OracleOp("clover", L, s["gauge"], clov=A[1], invclov=Ainv_e)
    po, co = F.qdp_spinor_cb(psi, 1), F.qdp_spinor_cb(chi, 1)
    if nrhs == 1:
        po, co = po[None], co[None]
    for k in range(nrhs):
        r = co[k] - O.apply(po[k], 1, 1)
        assert np.linalg.norm(r) / np.linalg.norm(co[k]) < tol, (inv, solver, k)
    rel = res.rel_resid if nrhs > 1 else [res.rel_resid]
    assert max(rel) < tol and res.n_count > 0
    solve.close()


def test_chroma_refuses_unconverged(api, setup):
    from qphix_b200 import chroma
    xml = XML.format(inv="QPHIX_CLOVER_INVERTER", solver="BICGSTAB", inner="h", maxit=3, tolf=5.0)
    solve = chroma.lin_op_sys_solver(xml, DIMS, F.qdp_gauge(setup["gauge"]))
    chi = F.qdp_spinor(F.gaussian_spinor(DIMS, 1), F.gaussian_spinor(DIMS, 2))
    psi = np.zeros_like(chi)
    with pytest.raises(RuntimeError, match="RsdToleranceFactor"):
        solve(psi, chi)
    assert np.all(psi == 0)
    solve.close()

