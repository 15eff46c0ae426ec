"""Chroma-facing layer on the CPU: <InvertParam> parsing and the derived
operator parameters (clover coefficients, diagonal mass and Dslash
anisotropy factors as the reference's tests/clover_term_qdp_w.h:120-142 and
tests/testNDTMvsTMCloverFull.cc:163-166 derive them), and the QDP++ CB2
array helpers."""
import numpy as np
import pytest

from qphix_b200 import chroma
from qphix_b200 import fields as F

XML = """<InvertParam>
  <invType>{inv}</invType>
  <SolverType>{solver}</SolverType>
  <MaxIter>500</MaxIter>
  <RsdTarget>1.0e-9</RsdTarget>
  <Delta>0.05</Delta>
  <CloverParams>
    {mass}
    <clovCoeffR>1.5</clovCoeffR>
    <clovCoeffT>0.8</clovCoeffT>
    <AnisoParam><anisoP>{aniso}</anisoP><t_dir>3</t_dir><xi_0>2.5</xi_0><nu>0.9</nu></AnisoParam>
  </CloverParams>
  <AntiPeriodicT>true</AntiPeriodicT>
  <NCores>8</NCores><By>4</By><Bz>4</Bz><PadXY>1</PadXY>
  <RsdToleranceFactor>10.0</RsdToleranceFactor>
  <Tune>false</Tune>
  <InnerType>f</InnerType>
</InvertParam>"""


def _xml(inv="QPHIX_CLOVER_INVERTER", solver="BICGSTAB", mass="<Kappa>0.12</Kappa>", aniso="true"):
    return XML.format(inv=inv, solver=solver, mass=mass, aniso=aniso)


def test_parse_and_derived_parameters():
    p = chroma.read_invert_param(_xml())
    assert p.invType == "QPHIX_CLOVER_INVERTER" and p.SolverType == "BICGSTAB"
    assert p.MaxIter == 500 and p.RsdTarget == 1e-9 and p.Delta == 0.05
    assert p.AntiPeriodicT and not p.Tune and p.RsdToleranceFactor == 10.0
    assert p.blocking == {"NCores": 8, "By": 4, "Bz": 4, "PadXY": 1}
    c = p.clover
    assert c.Mass == pytest.approx(1 / 0.24 - 4)
    ff = 0.9 / 2.5
    assert c.diag_mass() == pytest.approx(1 + 3 * ff + c.Mass)
    assert c.clover_coeffs() == pytest.approx((1.5 / 2.5, 0.8))
    assert c.aniso_factors() == pytest.approx((ff, 1.0))
    iso = chroma.read_invert_param(_xml(mass="<Mass>0.1</Mass>", aniso="false")).clover
    assert iso.diag_mass() == pytest.approx(4.1)
    assert iso.clover_coeffs() == (1.5, 0.8) and iso.aniso_factors() == (1.0, 1.0)


def test_clov_coeff_fills_both():
    x = _xml().replace("<clovCoeffR>1.5</clovCoeffR>", "<clovCoeff>1.7</clovCoeff>").replace(
        "<clovCoeffT>0.8</clovCoeffT>", "")
    c = chroma.read_invert_param(x).clover
    assert (c.clovCoeffR, c.clovCoeffT) == (1.7, 1.7)


def test_nested_invert_param():
    p = chroma.read_invert_param("<Prop><Param>" + _xml(inv="QPHIX_CLOVER_ITER_REFINE_BICGSTAB_INVERTER")
                                 + "</Param></Prop>")
    assert p.invType == "QPHIX_CLOVER_ITER_REFINE_BICGSTAB_INVERTER" and p.InnerType == "f"


@pytest.mark.parametrize("bad", [
    _xml(inv="QUDA_CLOVER_INVERTER"),
    _xml(solver="GMRES"),
    _xml(inv="QPHIX_CLOVER_ITER_REFINE_BICGSTAB_INVERTER", solver="CG"),
    _xml(mass="<Mass>0.1</Mass><Kappa>0.12</Kappa>"),
    _xml(mass=""),
    _xml().replace("<t_dir>3</t_dir>", "<t_dir>2</t_dir>"),
    _xml().replace("<InnerType>f</InnerType>", "<InnerType>x</InnerType>"),
])
def test_rejects(bad):
    with pytest.raises(ValueError):
        chroma.read_invert_param(bad)


def test_qdp_helpers():
    dims = (4, 4, 4, 8)
    e, o = F.gaussian_spinor(dims, 1), F.gaussian_spinor(dims, 2)
    full = F.qdp_spinor(e, o)
    assert full.shape == (2 * F.vh(dims), 4, 3)
    assert np.array_equal(F.qdp_spinor_cb(full, 0), e) and np.array_equal(F.qdp_spinor_cb(full, 1), o)
    g = F.make_gauge(dims, 3)
    q = F.qdp_gauge(g)
    vh = F.vh(dims)
    for mu in range(4):
        for cb in range(2):
            assert np.array_equal(q[mu, cb * vh:(cb + 1) * vh], g[cb, mu])
    packed = F.make_clover(dims, g, 0.1, 1.0)
    tri = F.qdp_clover(packed)
    assert tri.shape == (2 * vh, 72)
    site = tri[vh + 5]  # odd checkerboard, cb index 5
    for b in range(2):
        assert np.array_equal(site[b * 6:(b + 1) * 6], packed[1, 5, b, :6])
        assert np.array_equal(site[12 + 30 * b:12 + 30 * (b + 1)], packed[1, 5, b, 6:])
