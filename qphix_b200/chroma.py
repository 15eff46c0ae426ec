"""Chroma-facing caller layer: the QPhiX LinOpSysSolver that Chroma's
propagator applications select with an <InvertParam> block (the reference's
README.markdown, "Integration with Chroma" / "XML Drivers").

Given QDP++ fields -- links as multi1d<LatticeColorMatrix> and sources /
solutions as LatticeFermion, full-lattice arrays in QDP++'s checkerboarded
(CB2) site order, which the reference's packers read
(include/qphix/qdp_packer_parscalar.h:51-129) -- the solver

  * uploads the links straight from that order to the device (no QPhiX
    blocked host copy),
  * builds the clover term A on both checkerboards on the device from the
    links (clover-leaf field strength; coefficients and diagonal mass as the
    reference's tests/clover_term_qdp_w.h:114-188 derive them from
    CloverFermActParams, anisotropy included) and A_ee^-1,
  * solves the even-odd preconditioned system
    (A_oo - 1/4 D_oe A_ee^-1 D_eo) psi_o = chi_o on the odd checkerboard
    with the solver the XML names, and writes psi's odd checkerboard,
  * recomputes the true residual and refuses a result whose relative
    residual exceeds RsdToleranceFactor * RsdTarget, as Chroma's QPhiX solver
    does.

invType                                           solver
QPHIX_CLOVER_INVERTER, SolverType BICGSTAB        InvBiCGStab (FP64)
QPHIX_CLOVER_INVERTER, SolverType CG              InvCG on M^+ M with source M^+ chi
QPHIX_CLOVER_ITER_REFINE_BICGSTAB_INVERTER        InvRichardsonMultiPrec, BiCGStab inner
                                                  solver in InnerType precision, Delta
QPHIX_CLOVER_MIXED_BICGSTAB_INVERTER (new)        BiCGStab with reliable updates in
                                                  InnerType precision, Delta

InnerType stands in for Chroma's configure-time --enable-qphix-solver-inner-type
(h = FP16 storage, f = FP32, d = FP64; bf16 / q16 / q16f32 also accepted).
The CPU blocking and threading tags (NCores, ThreadsPerCore, By, Bz, Sy, Sz,
PadXY, PadXYZ, MinCt) are read and kept but have no effect on the GPU;
Tune = true switches the Dslash launch-shape autotuner on (it is on by
default unless QPHIX_GPU_TUNE=0), false leaves the process setting alone.  Links are taken without
fermion boundary phases; AntiPeriodicT sets the Dslash time boundary to -1.
Several sources at once (a leading right-hand-side axis) are solved as one
batched multi-right-hand-side solve.
"""
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field

import numpy as np

from . import api

INVERTERS = ("QPHIX_CLOVER_INVERTER", "QPHIX_CLOVER_ITER_REFINE_BICGSTAB_INVERTER",
             "QPHIX_CLOVER_MIXED_BICGSTAB_INVERTER")
INNER = {"h": "f16", "f": "f32", "d": "f64", "half": "f16", "float": "f32", "double": "f64",
         "bf16": "bf16", "q16": "q16", "q16f32": "q16f32"}
_BLOCKING = ("NCores", "ThreadsPerCore", "By", "Bz", "Sy", "Sz", "PadXY", "PadXYZ", "MinCt")


@dataclass
class AnisoParam:
    """AnisoParam_t (reference tests/clover_fermact_params_w.h:13-27)"""
    anisoP: bool = False
    t_dir: int = 3
    xi_0: float = 1.0
    nu: float = 1.0


@dataclass
class CloverParams:
    """CloverFermActParams (tests/clover_fermact_params_w.h:31-44).  The
    reference's clover construction ignores u0; so does this one."""
    Mass: float = 0.0
    clovCoeffR: float = 0.0
    clovCoeffT: float = 0.0
    u0: float = 1.0
    anisoParam: AnisoParam = field(default_factory=AnisoParam)

    def spatial_factor(self):
        """nu / xi_0 when anisotropic, else 1 (tests/clover_term_qdp_w.h:139-142)"""
        a = self.anisoParam
        return a.nu / a.xi_0 if a.anisoP else 1.0

    def diag_mass(self):
        """1 + (Nd - 1) nu / xi_0 + Mass (tests/clover_term_qdp_w.h:142)"""
        return 1.0 + 3.0 * self.spatial_factor() + self.Mass

    def clover_coeffs(self):
        """(c_R, c_T) before the builder's factor 1/2: c_R / xi_0 when
        anisotropic (tests/clover_term_qdp_w.h:126-131)"""
        a = self.anisoParam
        return (self.clovCoeffR / a.xi_0 if a.anisoP else self.clovCoeffR), self.clovCoeffT

    def aniso_factors(self):
        """(aniso_fac_s, aniso_fac_t) of the Dslash: (nu / xi_0, 1), as the
        reference's tests derive them (tests/testNDTMvsTMCloverFull.cc:163-166)"""
        return self.spatial_factor(), 1.0


@dataclass
class InvertParam:
    invType: str = "QPHIX_CLOVER_INVERTER"
    SolverType: str = "BICGSTAB"
    MaxIter: int = 1000
    RsdTarget: float = 1e-7
    Delta: float = 0.1
    clover: CloverParams = field(default_factory=CloverParams)
    AntiPeriodicT: bool = False
    Verbose: bool = False
    RsdToleranceFactor: float = 5.0
    Tune: bool = False
    InnerType: str = "h"
    InnerMaxIter: int = 5000
    blocking: dict = field(default_factory=dict)


def _text(node, tag, default=None, conv=str):
    e = node.find(tag)
    if e is None or e.text is None:
        return default
    return conv(e.text.strip())


def _bool(s):
    if s.lower() in ("true", "1", "yes"):
        return True
    if s.lower() in ("false", "0", "no"):
        return False
    raise ValueError(f"not a boolean: {s!r}")


def kappa_to_mass(kappa):
    """Chroma's kappaToMass: 1 / (2 kappa) - Nd"""
    return 1.0 / (2.0 * kappa) - 4.0


def read_clover_params(node):
    a = node.find("AnisoParam")
    aniso = AnisoParam()
    if a is not None:
        aniso = AnisoParam(_text(a, "anisoP", False, _bool), _text(a, "t_dir", 3, int),
                           _text(a, "xi_0", 1.0, float), _text(a, "nu", 1.0, float))
        if aniso.anisoP and aniso.t_dir != 3:
            raise ValueError("only t_dir = 3 is supported (the Dslash's anisotropic direction is time)")
    has_mass, has_kappa = node.find("Mass") is not None, node.find("Kappa") is not None
    if has_mass and has_kappa:
        raise ValueError("CloverParams: give Mass or Kappa, not both")
    if not (has_mass or has_kappa):
        raise ValueError("CloverParams: Mass or Kappa is required")
    mass = _text(node, "Mass", conv=float) if has_mass else kappa_to_mass(_text(node, "Kappa", conv=float))
    c = _text(node, "clovCoeff", None, float)
    cr = _text(node, "clovCoeffR", c, float)
    ct = _text(node, "clovCoeffT", c, float)
    if cr is None or ct is None:
        raise ValueError("CloverParams: clovCoeff or clovCoeffR and clovCoeffT are required")
    return CloverParams(mass, cr, ct, _text(node, "u0", 1.0, float), aniso)


def read_invert_param(xml):
    """Parse an <InvertParam> block (a string or an Element)."""
    root = ET.fromstring(xml) if isinstance(xml, str) else xml
    if root.tag != "InvertParam":
        found = root.find(".//InvertParam")
        if found is None:
            raise ValueError("no InvertParam element")
        root = found
    p = InvertParam()
    p.invType = _text(root, "invType", p.invType)
    if p.invType not in INVERTERS:
        raise ValueError(f"unknown invType {p.invType}")
    p.SolverType = _text(root, "SolverType", p.SolverType).upper()
    if p.SolverType not in ("BICGSTAB", "CG"):
        raise ValueError(f"unsupported SolverType {p.SolverType}")
    if p.invType != "QPHIX_CLOVER_INVERTER" and p.SolverType != "BICGSTAB":
        raise ValueError(f"{p.invType} uses a BICGSTAB inner solver")
    p.MaxIter = _text(root, "MaxIter", p.MaxIter, int)
    p.RsdTarget = _text(root, "RsdTarget", p.RsdTarget, float)
    p.Delta = _text(root, "Delta", p.Delta, float)
    cp = root.find("CloverParams")
    if cp is None:
        raise ValueError("CloverParams is required")
    p.clover = read_clover_params(cp)
    p.AntiPeriodicT = _text(root, "AntiPeriodicT", False, _bool)
    p.Verbose = _text(root, "Verbose", False, _bool)
    p.RsdToleranceFactor = _text(root, "RsdToleranceFactor", p.RsdToleranceFactor, float)
    p.Tune = _text(root, "Tune", False, _bool)
    p.InnerType = _text(root, "InnerType", p.InnerType)
    if p.InnerType not in INNER:
        raise ValueError(f"unknown InnerType {p.InnerType}")
    p.InnerMaxIter = _text(root, "InnerMaxIter", p.InnerMaxIter, int)
    p.blocking = {k: _text(root, k, None, int) for k in _BLOCKING if root.find(k) is not None}
    return p


@dataclass
class SystemSolverResults:
    """Chroma's SystemSolverResults_t: iterations and the true residual
    |chi - M psi| on the odd checkerboard (per right-hand side), plus the
    relative residual"""
    n_count: int
    resid: float
    rel_resid: float
    infos: list


class QPhiXCloverSysSolver:
    """LinOpSysSolver over the even-odd clover operator.

    links: complex [4, V, 3, 3] (multi1d<LatticeColorMatrix>, CB2 order),
    complex128 or complex64; dims: (Nx, Ny, Nz, Nt)."""

    def __init__(self, param, dims, links, device=0):
        self.param = param = read_invert_param(param) if not isinstance(param, InvertParam) else param
        self.dims = tuple(dims)
        self.lat = lat = api.Lattice(self.dims, device)
        if param.Tune:
            api.tune_enable(True)
        u = lat.gauge("f64", 18).upload_qdp(links)
        cl = param.clover
        dm, (cr, ct) = cl.diag_mass(), cl.clover_coeffs()
        A = [lat.clover("f64") for _ in range(2)]
        for cb in (0, 1):  # api.clover_build takes the bare mass: diagonal 4 + mass
            api.clover_build(A[cb], u, cb, dm - 4.0, cr, ct)
        Ainv = lat.clover("f64")
        api.clover_invert(Ainv, A[0])
        self.fields = [u, A, Ainv]
        s, t = cl.aniso_factors()
        tb = -1.0 if param.AntiPeriodicT else 1.0
        u12 = lat.gauge("f64", 12).upload_qdp(links)
        self.M = api.EvenOddCloverOperator(u12, A[1], Ainv, tb, s, t)
        self.M_low = None
        if param.invType != "QPHIX_CLOVER_INVERTER":
            ip = INNER[param.InnerType]
            ul = lat.gauge(ip, 12).upload_qdp(links)
            Al, Ail = lat.clover(ip), lat.clover(ip)
            api.clover_convert(Al, A[1])
            api.clover_convert(Ail, Ainv)
            self.fields += [ul, Al, Ail]
            self.M_low = api.EvenOddCloverOperator(ul, Al, Ail, tb, s, t)

    def __call__(self, psi, chi):
        """Solve M psi_o = chi_o.  psi, chi: complex [(nrhs,) V, 4, 3] CB2
        full-lattice arrays; psi's odd checkerboard is written in place (its
        even one is left alone), and psi's odd checkerboard on entry is the
        initial guess."""
        p = self.param
        single = chi.ndim == 3
        nrhs = 1 if single else chi.shape[0]
        lat = self.lat
        b = lat.spinor("f64", nrhs).upload_qdp(chi, 1)
        x = lat.spinor("f64", nrhs).upload_qdp(psi, 1)
        if p.invType == "QPHIX_CLOVER_INVERTER" and p.SolverType == "CG":
            # M^+ M x = M^+ chi
            bd = lat.spinor("f64", nrhs)
            self.M(bd, b, -1, 1)
            infos = api.InvCG(self.M, p.MaxIter)(x, bd, p.RsdTarget)
        elif p.invType == "QPHIX_CLOVER_INVERTER":
            infos = api.InvBiCGStab(self.M, p.MaxIter)(x, b, p.RsdTarget)
        elif p.invType == "QPHIX_CLOVER_ITER_REFINE_BICGSTAB_INVERTER":
            infos = api.InvRichardsonMultiPrec(self.M, self.M_low, "bicgstab", p.Delta, p.MaxIter,
                                               p.InnerMaxIter)(x, b, p.RsdTarget)
        else:
            infos = api.InvBiCGStabMixed(self.M, self.M_low, p.Delta, p.MaxIter)(x, b, p.RsdTarget)
        # true residual of M psi = chi on the odd checkerboard
        r = lat.spinor("f64", nrhs)
        self.M(r, x, 1, 1)
        api.caxpby(1.0, b, -1.0, r)
        rn = np.sqrt(api.norm2(r))
        bn = np.sqrt(api.norm2(b))
        rel = rn / np.where(bn > 0, bn, 1.0)
        limit = p.RsdToleranceFactor * p.RsdTarget
        if np.any(rel > limit):
            raise RuntimeError(f"QPhiX clover solve: true relative residual {rel.max():.3e} exceeds "
                               f"RsdToleranceFactor * RsdTarget = {limit:.3e}")
        x.download_qdp(psi, 1)
        n = max(i["n_iters"] for i in infos)
        if single:
            return SystemSolverResults(n, float(rn[0]), float(rel[0]), infos)
        return SystemSolverResults(n, [float(v) for v in rn], [float(v) for v in rel], infos)

    def close(self):
        for f in (self.M, self.M_low):
            if f is not None:
                f.close()
        self.lat.close()


def lin_op_sys_solver(xml, dims, links, device=0):
    """Chroma's factory entry: an InvertParam XML block -> the solver"""
    return QPhiXCloverSysSolver(read_invert_param(xml), dims, links, device)


__all__ = ["AnisoParam", "CloverParams", "InvertParam", "SystemSolverResults", "QPhiXCloverSysSolver",
           "read_invert_param", "kappa_to_mass", "lin_op_sys_solver"]

