"""Python mirror of QPhiX's host interface over the C ABI.

Class and method names follow the reference (include/qphix/*.h) so that code
written against QPhiX reads the same:

  Geometry           -> Lattice (+ field allocators)      geometry.h:115
  Dslash             -> Dslash.dslash / dslashAChiMinusBDPsi / dslashDir
  ClovDslash         -> ClovDslash (+ clovMult)          clover_dslash_def.h:14
  TMDslash           -> TMDslash                          tm_dslash_def.h:11
  TMClovDslash       -> TMClovDslash                      tm_clov_dslash_def.h:11
  EvenOdd*Operator   -> EvenOddWilsonOperator, EvenOddCloverOperator,
                        EvenOddTMWilsonOperator, EvenOddTMCloverOperator
  InvCG / InvBiCGStab / InvMR / InvRichardsonMultiPrec / MInvCG

Fields are device-resident handles; `upload` / `download` move canonical
numpy arrays (see qphix_b200.fields) or QPhiX blocked host arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check

PREC = {"f64": L.F64, "f32": L.F32, "f16": L.F16, "bf16": L.BF16, "q16": L.Q16, "q16f32": L.Q16F32,
        "double": L.F64, "float": L.F32, "half": L.F16}


def lib():
    return L.load()


def _canon_layout():
    h = L.HostLayout()
    h.kind = L.HOST_CANONICAL
    h.ft = L.HOST_F64
    return h


def qphix_layout(veclen, soalen, compress12, ft="f64", pad_xy=0, pad_xyz=0):
    h = L.HostLayout()
    h.kind = L.HOST_QPHIX
    h.ft = {"f64": L.HOST_F64, "f32": L.HOST_F32, "f16": L.HOST_F16}[ft]
    h.veclen, h.soalen, h.compress12 = veclen, soalen, int(bool(compress12))
    h.pad_xy, h.pad_xyz = pad_xy, pad_xyz
    return h


def qdp_layout(cb=0, ft="f64"):
    """QDP++ / Chroma CB2 full-lattice arrays (the order the reference's
    qdp_pack_* read, include/qphix/qdp_packer_parscalar.h:51-230); spinor and
    clover transfers touch checkerboard cb only."""
    h = L.HostLayout()
    h.kind = L.HOST_QDP
    h.ft = {"f64": L.HOST_F64, "f32": L.HOST_F32}[ft]
    h.cb = cb
    return h


def _qdp_ft(a):
    if a.dtype in (np.complex128, np.float64):
        return "f64"
    if a.dtype in (np.complex64, np.float32):
        return "f32"
    raise TypeError(f"QDP arrays are FP64 or FP32, not {a.dtype}")


class Lattice:
    """One lattice (Geometry) with its own CUDA stream and reduction workspace."""

    def __init__(self, dims, device=0):
        lib()
        check(L._lib.qphix_gpu_init(device))
        self.dims = tuple(int(d) for d in dims)
        arr = (C.c_int * 4)(*self.dims)
        h = C.c_void_p()
        check(L._lib.qphix_gpu_lattice_create(arr, C.byref(h)))
        self.h = h
        self.vh = int(L._lib.qphix_gpu_lattice_volcb(h))

    def close(self):
        if getattr(self, "h", None):
            L._lib.qphix_gpu_lattice_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(L._lib.qphix_gpu_lattice_sync(self.h))

    def set_stream(self, stream_handle: int):
        check(L._lib.qphix_gpu_lattice_set_stream(self.h, C.c_void_p(stream_handle)))

    # allocators (Geometry::allocCB*)
    def spinor(self, prec="f64", nrhs=1):
        return Field(self, L.SPINOR, PREC[prec], 0, nrhs)

    def gauge(self, prec="f64", recon=18):
        return Field(self, L.GAUGE, PREC[prec], recon, 1)

    def clover(self, prec="f64"):
        return Field(self, L.CLOVER, PREC[prec], 0, 1)

    def full_clover(self, prec="f64"):
        return Field(self, L.FULLCLOVER, PREC[prec], 0, 1)


class Field:
    def __init__(self, lat: Lattice, kind, prec, recon, nrhs):
        self.lat, self.kind, self.prec, self.recon, self.nrhs = lat, kind, prec, recon, nrhs
        h = C.c_void_p()
        check(L._lib.qphix_gpu_field_create(lat.h, kind, prec, recon, nrhs, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            L._lib.qphix_gpu_field_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nbytes(self):
        n = C.c_size_t()
        check(L._lib.qphix_gpu_field_bytes(self.h, C.byref(n)))
        return n.value

    # ---- canonical numpy arrays -------------------------------------------------
    def upload(self, arr, rhs=-1):
        """Fill from a canonical array (complex spinor [(nrhs,) Vh, 4, 3];
        complex gauge [2, 4, Vh, 3, 3]; packed clover float [Vh, 2, 36];
        complex full clover [Vh, 2, 6, 6])."""
        a = np.asarray(arr)
        if np.iscomplexobj(a):
            a = np.stack([a.real, a.imag], axis=-1)
        a = np.ascontiguousarray(a, dtype=np.float64)
        cb = -1
        check(L._lib.qphix_gpu_field_upload(self.h, a.ctypes.data_as(C.c_void_p),
                                            C.byref(_canon_layout()), cb, rhs))
        return self

    def download(self, rhs=-1):
        if self.kind == L.SPINOR:
            n = self.nrhs if rhs < 0 else 1
            out = np.empty((n, self.lat.vh, 4, 3, 2))
            check(L._lib.qphix_gpu_field_download(self.h, out.ctypes.data_as(C.c_void_p),
                                                  C.byref(_canon_layout()), rhs))
            c = out[..., 0] + 1j * out[..., 1]
            return c[0] if (rhs >= 0 or self.nrhs == 1) else c
        nr = 72 if self.kind == L.CLOVER else 144
        out = np.empty((self.lat.vh, nr))
        check(L._lib.qphix_gpu_field_download(self.h, out.ctypes.data_as(C.c_void_p),
                                              C.byref(_canon_layout()), -1))
        return out

    # ---- QPhiX blocked host arrays (drop-in path) ------------------------------
    def upload_qphix(self, arr, layout, cb=-1, rhs=-1):
        a = np.ascontiguousarray(arr)
        check(L._lib.qphix_gpu_field_upload(self.h, a.ctypes.data_as(C.c_void_p), C.byref(layout),
                                            cb, rhs))
        return self

    def download_qphix(self, out, layout, rhs=-1):
        assert out.flags["C_CONTIGUOUS"]
        check(L._lib.qphix_gpu_field_download(self.h, out.ctypes.data_as(C.c_void_p),
                                              C.byref(layout), rhs))
        return out

    # ---- QDP++ / Chroma CB2 full-lattice arrays ---------------------------------
    def upload_qdp(self, arr, cb=0, rhs=-1):
        """spinor complex [(nrhs,) V, 4, 3] (checkerboard cb of it), gauge complex
        [4, V, 3, 3] (both checkerboards), clover float [V, 72] in Chroma's
        triangle order (checkerboard cb); complex128 / float64 or complex64 /
        float32."""
        a = np.ascontiguousarray(arr)
        lay = qdp_layout(cb if self.kind != L.GAUGE else 0, _qdp_ft(a))
        check(L._lib.qphix_gpu_field_upload(self.h, a.ctypes.data_as(C.c_void_p), C.byref(lay), -1, rhs))
        return self

    def download_qdp(self, out, cb, rhs=-1):
        """write checkerboard cb of a full-lattice spinor / clover array in place"""
        assert out.flags["C_CONTIGUOUS"]
        check(L._lib.qphix_gpu_field_download(self.h, out.ctypes.data_as(C.c_void_p),
                                              C.byref(qdp_layout(cb, _qdp_ft(out))), rhs))
        return out

    def convert_from(self, src, scale=1.0):
        check(L._lib.qphix_gpu_field_convert(self.h, src.h, scale))
        return self


# ---------------------------------------------------------------------------
# operator parameters and the Dslash family
# ---------------------------------------------------------------------------


def op_params(kind, t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0, use_tbc=None, tbc_phases=None,
              mass=0.0, twisted_mass=0.0, prec_mass_rho=0.0, epsilon=0.0):
    p = L.OpParams()
    p.kind = kind
    p.t_boundary = t_boundary
    p.aniso_s = aniso_s
    p.aniso_t = aniso_t
    for d in range(4):
        p.tbc_phases[d][0] = 1.0
        p.tbc_phases[d][1] = 0.0
    if use_tbc is not None and tbc_phases is not None:
        for d in range(4):
            p.use_tbc[d] = int(bool(use_tbc[d]))
            p.tbc_phases[d][0] = tbc_phases[d][0]
            p.tbc_phases[d][1] = tbc_phases[d][1]
    p.mass = mass
    p.twisted_mass = twisted_mass
    p.prec_mass_rho = prec_mass_rho
    p.epsilon = epsilon
    return p


def _h(f):
    return None if f is None else f.h


class Dslash:
    """include/qphix/dslash_def.h:27-58"""

    kind = L.WILSON

    def __init__(self, lat, t_boundary, aniso_s, aniso_t, use_tbc=None, tbc_phases=None, **kw):
        self.lat = lat
        self.p = op_params(self.kind, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases, **kw)

    def dslash(self, res, psi, u, isign, cb):
        check(L._lib.qphix_gpu_dslash(C.byref(self.p), res.h, psi.h, u.h, None, None, isign, cb))

    def dslashAChiMinusBDPsi(self, res, psi, chi, u, alpha, beta, isign, cb):
        check(L._lib.qphix_gpu_dslash_achimbdpsi(C.byref(self.p), res.h, psi.h, chi.h, u.h, None,
                                                 alpha, beta, isign, cb, 1.0))

    def dslashDir(self, res, psi, u, cb, d):
        check(L._lib.qphix_gpu_dslash_dir(C.byref(self.p), res.h, psi.h, u.h, cb, d))


class ClovDslash(Dslash):
    """include/qphix/clover_dslash_def.h:24-53"""

    kind = L.CLOVER_OP

    def __init__(self, lat, t_boundary, aniso_s, aniso_t, use_tbc=None, tbc_phases=None,
                 prec_mass_rho=0.0):
        super().__init__(lat, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases,
                         prec_mass_rho=prec_mass_rho)

    def dslash(self, res, psi, u, invclov, isign, cb):
        check(L._lib.qphix_gpu_dslash(C.byref(self.p), res.h, psi.h, u.h, invclov.h, None, isign, cb))

    def dslashAChiMinusBDPsi(self, res, psi, chi, u, clov, beta, isign, cb):
        check(L._lib.qphix_gpu_dslash_achimbdpsi(C.byref(self.p), res.h, psi.h, chi.h, u.h, clov.h,
                                                 0.0, beta, isign, cb, 1.0))

    def clovMult(self, res, chi, clov):
        check(L._lib.qphix_gpu_clover_apply(res.h, chi.h, clov.h))

    def dslashAChiMinusBDPsiNorms(self, res, psi, chi, u, clov, beta, isign, cb, w=None, fetch=True):
        """dslashAChiMinusBDPsi with its fused reductions (the solvers'
        launch): per rhs [|res|^2, (<w,res> re, im,) <res,chi> re, im], or
        None with fetch=False (values stay on the device)."""
        nval = 5 if w is not None else 3
        out = np.zeros(res.nrhs * nval) if fetch else None
        check(L._lib.qphix_gpu_dslash_achimbdpsi_norms(
            C.byref(self.p), res.h, psi.h, chi.h, u.h, clov.h, 0.0, beta, isign, cb, 1.0,
            w.h if w is not None else None, out.ctypes.data if fetch else None))
        return out.reshape(res.nrhs, nval) if fetch else None


class TMDslash(Dslash):
    """include/qphix/tm_dslash_def.h:23-49"""

    kind = L.TM

    def __init__(self, lat, t_boundary, aniso_s, aniso_t, mass, twisted_mass, use_tbc=None,
                 tbc_phases=None):
        super().__init__(lat, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases, mass=mass,
                         twisted_mass=twisted_mass)

    def dslashAChiMinusBDPsi(self, res, psi, chi, u, alpha, beta, isign, cb, musign=1.0):
        check(L._lib.qphix_gpu_dslash_achimbdpsi(C.byref(self.p), res.h, psi.h, chi.h, u.h, None,
                                                 alpha, beta, isign, cb, musign))


class TMClovDslash(Dslash):
    """include/qphix/tm_clov_dslash_def.h:30-66"""

    kind = L.TMCLOVER

    def __init__(self, lat, t_boundary, aniso_s, aniso_t, use_tbc=None, tbc_phases=None,
                 prec_mass_rho=0.0):
        super().__init__(lat, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases,
                         prec_mass_rho=prec_mass_rho)

    def dslash(self, res, psi, u, invclov, isign, cb):
        check(L._lib.qphix_gpu_dslash(C.byref(self.p), res.h, psi.h, u.h, invclov[0].h, invclov[1].h,
                                      isign, cb))

    def dslashAChiMinusBDPsi(self, res, psi, chi, u, clov, beta, isign, cb):
        check(L._lib.qphix_gpu_dslash_achimbdpsi(C.byref(self.p), res.h, psi.h, chi.h, u.h, clov.h,
                                                 0.0, beta, isign, cb, 1.0))


# ---------------------------------------------------------------------------
# clover term on the device
# ---------------------------------------------------------------------------


def clover_build(clov, gauge, cb, mass, csw, csw_t=None):
    """A = (4 + mass) + sigma.F (clover leaf, c_sw) on checkerboard cb."""
    check(L._lib.qphix_gpu_clover_build(clov.h, gauge.h, cb, 4.0 + mass, csw, csw if csw_t is None else csw_t))
    return clov


def clover_invert(dst, src):
    check(L._lib.qphix_gpu_clover_invert(dst.h, src.h))
    return dst


def clover_invert_twisted(dst_plus, dst_minus, src, mu):
    check(L._lib.qphix_gpu_clover_invert_twisted(dst_plus.h, dst_minus.h, src.h, mu))
    return dst_plus, dst_minus


def clover_invert_ndtm(finv_up, finv_dn, clov_odiag, src, mu, eps):
    """the two-flavour inverses of EvenOddNDTMCloverReuseOperator
    (ndtm_reuse_operator_clover.h:38-50): Q (A -/+ i mu g5) and eps Q,
    Q = (A^2 + mu^2 - eps^2)^-1"""
    check(L._lib.qphix_gpu_clover_invert_ndtm(finv_up.h, finv_dn.h, clov_odiag.h, src.h, mu, eps))
    return finv_up, finv_dn, clov_odiag


def clover_convert(dst, src):
    check(L._lib.qphix_gpu_clover_convert(dst.h, src.h))
    return dst


# ---------------------------------------------------------------------------
# even-odd operators
# ---------------------------------------------------------------------------


class EvenOddLinearOperator:
    """include/qphix/linearOp.h:9-92: operator()(res, in, isign, target_cb=1)"""

    def __init__(self, p, gauge, clov=None, invclov=None, finv=(None, None)):
        self.p = p
        self.fields = (gauge, clov, invclov, finv)
        h = C.c_void_p()
        check(L._lib.qphix_gpu_eo_op_create(C.byref(p), gauge.h, _h(clov), _h(invclov), _h(finv[0]),
                                            _h(finv[1]), C.byref(h)))
        self.h = h
        self.lat = gauge.lat

    def __call__(self, res, inp, isign=1, target_cb=1):
        check(L._lib.qphix_gpu_eo_op_apply(self.h, res.h, inp.h, isign, target_cb))

    def M_offdiag(self, res, inp, isign, target_cb):
        """checkerboard off-diagonal block; only the Wilson and clover operators
        have it (the reference's twisted-mass operators print "not yet
        implemented", twisted_mass.h:79-87)"""
        raise NotImplementedError(f"M_offdiag not implemented for {type(self).__name__}")

    def M_diag_inv(self, res, inp, isign, cb=0):
        """inverse of the checkerboard-diagonal block (Wilson and clover only)"""
        raise NotImplementedError(f"M_diag_inv not implemented for {type(self).__name__}")

    def _offdiag(self, res, inp, isign, target_cb):
        # -1/2 D onto target_cb (wilson.h:68-77, clover.h:175-184)
        w = L.OpParams.from_buffer_copy(self.p)
        w.kind = L.WILSON
        check(L._lib.qphix_gpu_dslash(C.byref(w), res.h, inp.h, self.fields[0].h, None, None, isign,
                                      target_cb))
        caxpby(0.0, res, -0.5, res)

    def close(self):
        if getattr(self, "h", None):
            L._lib.qphix_gpu_eo_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EvenOddWilsonOperator(EvenOddLinearOperator):
    """include/qphix/wilson.h:20-40"""

    def __init__(self, mass, u, t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0, use_tbc=None,
                 tbc_phases=None):
        super().__init__(op_params(L.WILSON, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases,
                                   mass=mass), u)
        self.mass = mass

    def M_offdiag(self, res, inp, isign, target_cb):
        self._offdiag(res, inp, isign, target_cb)

    def M_diag_inv(self, res, inp, isign, cb=0):
        """1 / (4 + m) (wilson.h:79-86)"""
        copy(res, inp)
        caxpby(0.0, res, 1.0 / (4.0 + self.mass), res)


class EvenOddCloverOperator(EvenOddLinearOperator):
    """include/qphix/clover.h:31-102 (clov = A_oo, invclov = A_ee^-1; invclov_odd =
    A_oo^-1, needed only by M_diag_inv on the odd checkerboard)"""

    def __init__(self, u, clov, invclov, t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0, use_tbc=None,
                 tbc_phases=None, prec_mass_rho=0.0, invclov_odd=None):
        super().__init__(op_params(L.CLOVER_OP, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases,
                                   prec_mass_rho=prec_mass_rho), u, clov, invclov)
        self.invclov = (invclov, invclov_odd)

    def M_offdiag(self, res, inp, isign, target_cb):
        self._offdiag(res, inp, isign, target_cb)

    def M_diag_inv(self, res, inp, isign, cb=0):
        """A^-1 of checkerboard cb (clover.h:186-192)"""
        ai = self.invclov[cb]
        if ai is None:
            raise ValueError("M_diag_inv: no inverse clover term for this checkerboard")
        check(L._lib.qphix_gpu_clover_apply(res.h, inp.h, ai.h))


class EvenOddTMWilsonOperator(EvenOddLinearOperator):
    """include/qphix/twisted_mass.h:22-46"""

    def __init__(self, mass, twisted_mass, u, t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0,
                 use_tbc=None, tbc_phases=None):
        super().__init__(op_params(L.TM, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases,
                                   mass=mass, twisted_mass=twisted_mass), u)


class EvenOddNDTMWilsonOperator(EvenOddLinearOperator):
    """include/qphix/ndtm_reuse_operator.h:16-110 (EvenOddNDTMWilsonReuseOperator):
    the two-flavour twisted-mass operator.  Its fields hold (up, down) pairs
    as right-hand sides 2k, 2k + 1 (a spinor field of nrhs = 2 is one doublet);
    InvCG solves each pair as one system."""

    def __init__(self, mass, twisted_mass, epsilon, u, t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0):
        super().__init__(op_params(L.NDTM, t_boundary, aniso_s, aniso_t, None, None, mass=mass,
                                   twisted_mass=twisted_mass, epsilon=epsilon), u)


class EvenOddNDTMCloverOperator(EvenOddLinearOperator):
    """include/qphix/ndtm_reuse_operator_clover.h:23-165
    (EvenOddNDTMCloverReuseOperator): the two-flavour twisted-mass clover
    operator; clov = A of the target checkerboard, invclov_odiag and
    invclov = (up, down) the inverses of the other checkerboard's two-flavour
    block (clover_invert_ndtm).  Fields hold (up, down) pairs as for
    EvenOddNDTMWilsonOperator."""

    def __init__(self, twisted_mass, epsilon, u, clov, invclov_odiag, invclov, t_boundary=-1.0,
                 aniso_s=1.0, aniso_t=1.0):
        super().__init__(op_params(L.NDTMCLOVER, t_boundary, aniso_s, aniso_t, None, None,
                                   twisted_mass=twisted_mass, epsilon=epsilon), u, clov, invclov_odiag,
                         tuple(invclov))


class TMClovDslashTwoFlav:
    """The two-flavour members of TMClovDslash (tm_clov_dslash_def.h:76-110):
    the Wilson hop followed by the two-flavour inverse clover term, and
    two_flav_AChiMinusBDPsi."""

    def __init__(self, lat, t_boundary, aniso_s, aniso_t, twisted_mass, epsilon):
        self.lat = lat
        self.p = op_params(L.NDTMCLOVER, t_boundary, aniso_s, aniso_t, twisted_mass=twisted_mass,
                           epsilon=epsilon)

    def dslash_inverse_clover(self, res, psi, u, invclov, invclov_odiag, isign, cb):
        check(L._lib.qphix_gpu_dslash_two_flav_clover(C.byref(self.p), res.h, psi.h, u.h, invclov[0].h,
                                                      invclov[1].h, invclov_odiag.h, isign, cb))

    def two_flav_inverse_clover_term(self, res, psi, invclov, invclov_odiag, isign):
        """the inverse clover term alone (tm_clov_dslash_def.h:96-110)"""
        check(L._lib.qphix_gpu_two_flav_clover_apply(res.h, psi.h, invclov[0].h, invclov[1].h, invclov_odiag.h,
                                                     isign))

    def two_flav_AChiMinusBDPsi(self, res, psi, chi, u, clov, beta, isign, cb):
        check(L._lib.qphix_gpu_dslash_achimbdpsi(C.byref(self.p), res.h, psi.h, chi.h, u.h, clov.h, 0.0,
                                                 beta, isign, cb, 1.0))


class EvenOddTMCloverOperator(EvenOddLinearOperator):
    """include/qphix/twisted_mass_clover.h:29-73 (invclov = [(A+i mu g5)^-1, (A-i mu g5)^-1])"""

    def __init__(self, u, clov, invclov, t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0, use_tbc=None,
                 tbc_phases=None, prec_mass_rho=0.0):
        super().__init__(op_params(L.TMCLOVER, t_boundary, aniso_s, aniso_t, use_tbc, tbc_phases,
                                   prec_mass_rho=prec_mass_rho), u, clov, None, tuple(invclov))


# ---------------------------------------------------------------------------
# solvers
# ---------------------------------------------------------------------------


def _infos(n):
    return (L.SolveInfo * n)()


def _as_dicts(infos):
    return [dict(n_iters=i.n_iters, rsd_sq_final=i.rsd_sq_final, site_flops=i.site_flops,
                 mv_apps=i.mv_apps, status=i.status, true_rel_resid=i.true_rel_resid,
                 seconds=i.seconds) for i in infos]


def _solve_rc(rc):
    # non-convergence and breakdown are reported through info, like the reference
    if rc not in (L.OK, L.ENOTCONV, L.EBREAKDOWN):
        check(rc)


class InvCG:
    """include/qphix/invcg.h:31-88"""

    def __init__(self, M, max_iters):
        self.M, self.max_iters = M, max_iters

    def __call__(self, x, rhs, rsd_target, isign=1, cb=1):
        inf = _infos(x.nrhs)
        _solve_rc(L._lib.qphix_gpu_solve_cg(self.M.h, x.h, rhs.h, rsd_target, self.max_iters, isign,
                                            cb, inf))
        return _as_dicts(inf)


class InvBiCGStab(InvCG):
    """include/qphix/invbicgstab.h:24-80"""

    def __call__(self, x, rhs, rsd_target, isign=1, cb=1):
        inf = _infos(x.nrhs)
        _solve_rc(L._lib.qphix_gpu_solve_bicgstab(self.M.h, x.h, rhs.h, rsd_target, self.max_iters,
                                                  isign, cb, inf))
        return _as_dicts(inf)


class InvMR:
    """include/qphix/invmr.h:249-300"""

    def __init__(self, M, max_iters, omega=1.0):
        self.M, self.max_iters, self.omega = M, max_iters, omega

    def __call__(self, x, rhs, rsd_target, isign=1, cb=1):
        inf = _infos(x.nrhs)
        _solve_rc(L._lib.qphix_gpu_solve_mr(self.M.h, x.h, rhs.h, rsd_target, self.max_iters,
                                            self.omega, isign, cb, inf))
        return _as_dicts(inf)


class InvMRSmoother:
    """include/qphix/invmr.h:302-354: a fixed number of MR iterations"""

    def __init__(self, M, max_iters, omega=1.0):
        self.M, self.max_iters, self.omega = M, max_iters, omega

    def __call__(self, x, rhs, rsd_target=0.0, isign=1, cb=1):
        inf = _infos(x.nrhs)
        _solve_rc(L._lib.qphix_gpu_solve_mr_smoother(self.M.h, x.h, rhs.h, self.max_iters, self.omega,
                                                     isign, cb, inf))
        return _as_dicts(inf)


class InvRichardsonMultiPrec:
    """include/qphix/inv_richardson_multiprec.h:22-42 (inner solver on op_inner)"""

    INNER = {"cg": L.SOLVER_CG, "bicgstab": L.SOLVER_BICGSTAB, "mr": L.SOLVER_MR}

    def __init__(self, M_outer, M_inner, inner="bicgstab", delta=0.1, max_iters=100,
                 inner_max_iters=5000):
        self.Mo, self.Mi = M_outer, M_inner
        self.inner = self.INNER[inner]
        self.delta, self.max_iters, self.inner_max = delta, max_iters, inner_max_iters

    def __call__(self, x, rhs, rsd_target, isign=1, cb=1):
        inf = _infos(x.nrhs)
        _solve_rc(L._lib.qphix_gpu_solve_richardson(self.Mo.h, self.Mi.h, self.inner, x.h, rhs.h,
                                                    rsd_target, self.delta, self.max_iters,
                                                    self.inner_max, isign, cb, inf))
        return _as_dicts(inf)


class FullSpinor:
    """include/qphix/full_spinor.h: both checkerboards of a spinor field"""

    def __init__(self, lat, prec="f64", nrhs=1):
        self.cbs = (lat.spinor(prec, nrhs), lat.spinor(prec, nrhs))

    def getCBData(self, cb):
        return self.cbs[cb]


class UnprecSolverWrapper:
    """include/qphix/unprec_solver_wrapper.h:17-99 with the driver of
    include/qphix/abs_solver.h:271-438 (AbstractUnprecSolver): solves the
    unpreconditioned M x = b with an even-odd solver on solve_cb.

      b'      = b_cb - M_offdiag(M_diag_inv(b_other), solve_cb)
      x_cb    = eo_solver(b')
      x_other = M_diag_inv(b_other - M_offdiag(x_cb, other))

    The prepared source lives in x's other checkerboard, as in the reference.
    M_diag_inv is called with its default checkerboard (unprec_solver_wrapper.h:
    54,84): the inverse diagonal block M was built with, i.e. that of the
    checkerboard not solved for (an operator for solve_cb = 0 holds A_ee as
    clov and A_oo^-1 as invclov)."""

    def __init__(self, eo_solver, M):
        self.solver, self.M = eo_solver, M

    def getEOSolver(self):
        return self.solver

    @staticmethod
    def _tmp(like):
        return Field(like.lat, L.SPINOR, like.prec, 0, like.nrhs)

    def SourcePrepare(self, out, in_cb, in_other_cb, isign, solve_cb):
        t1, t2 = self._tmp(in_cb), self._tmp(in_cb)
        self.M.M_diag_inv(t1, in_other_cb, isign)
        self.M.M_offdiag(t2, t1, isign, solve_cb)
        copy(out, in_cb)
        caxpby(-1.0, t2, 1.0, out)

    def SolutionReconstruct(self, out_other_cb, in_other_cb, out_cb, isign, solve_cb):
        t1, t2 = self._tmp(out_cb), self._tmp(out_cb)
        self.M.M_offdiag(t1, out_cb, isign, 1 - solve_cb)
        copy(t2, in_other_cb)
        caxpby(-1.0, t1, 1.0, t2)
        self.M.M_diag_inv(out_other_cb, t2, isign)

    def __call__(self, x, rhs, rsd_target, isign=1, solve_cb=1):
        o = 1 - solve_cb
        self.SourcePrepare(x.getCBData(o), rhs.getCBData(solve_cb), rhs.getCBData(o), isign, solve_cb)
        infos = self.solver(x.getCBData(solve_cb), x.getCBData(o), rsd_target, isign, solve_cb)
        self.SolutionReconstruct(x.getCBData(o), rhs.getCBData(o), x.getCBData(solve_cb), isign, solve_cb)
        return infos


class InvBiCGStabMixed:
    """BiCGStab with reliable updates: iterations on M_low, true residuals and
    the solution on M (no counterpart in the reference)."""

    def __init__(self, M, M_low, delta=0.1, max_iters=10000):
        self.M, self.Ml, self.delta, self.max_iters = M, M_low, delta, max_iters

    def __call__(self, x, rhs, rsd_target, isign=1, cb=1):
        inf = _infos(x.nrhs)
        _solve_rc(L._lib.qphix_gpu_solve_bicgstab_mixed(self.M.h, self.Ml.h, x.h, rhs.h, rsd_target,
                                                        self.delta, self.max_iters, isign, cb, inf))
        return _as_dicts(inf)


class MInvCG:
    """include/qphix/minvcg.h:23-77"""

    def __init__(self, M, max_iters, max_shifts=32):
        self.M, self.max_iters, self.max_shifts = M, max_iters, max_shifts

    def __call__(self, xs, rhs, shifts, rsd_targets, isign=1, cb=1):
        n = len(shifts)
        if n > self.max_shifts:
            raise ValueError("too many shifts")
        xh = (C.c_void_p * n)(*[x.h.value for x in xs])
        sh = np.ascontiguousarray(shifts, dtype=np.float64)
        rs = np.ascontiguousarray(rsd_targets, dtype=np.float64)
        fin = np.zeros(n)
        it = C.c_int(0)
        mv = C.c_ulong(0)
        check(L._lib.qphix_gpu_solve_mshift_cg(self.M.h, C.cast(xh, L.PP), rhs.h, n,
                                               sh.ctypes.data_as(C.c_void_p),
                                               rs.ctypes.data_as(C.c_void_p), self.max_iters, isign,
                                               cb, C.byref(it), fin.ctypes.data_as(C.c_void_p),
                                               C.byref(mv)))
        return it.value, fin, mv.value


class InvCGShifted(InvCG):
    """CG on (M^+M + shifts[i]) x_i = rhs_i, one shift per right-hand side of
    the block (qphix_gpu_solve_cg_shifted; no reference counterpart)."""

    def __call__(self, x, rhs, shifts, rsd_targets, isign=1, cb=1):
        inf = _infos(x.nrhs)
        sh = np.ascontiguousarray(np.broadcast_to(shifts, (x.nrhs,)), dtype=np.float64)
        rs = np.ascontiguousarray(np.broadcast_to(rsd_targets, (x.nrhs,)), dtype=np.float64)
        _solve_rc(L._lib.qphix_gpu_solve_cg_shifted(self.M.h, x.h, rhs.h, sh.ctypes.data_as(C.c_void_p),
                                                    rs.ctypes.data_as(C.c_void_p), self.max_iters, isign,
                                                    cb, inf))
        return _as_dicts(inf)


class MInvCGMixed:
    """Multishift CG with low-precision iterations and a batched refinement of
    every shift to its target (qphix_gpu_solve_mshift_cg_mixed; no reference
    counterpart).  xs: one-rhs fields in M's precision; M_low: the same
    operator on low-precision fields."""

    def __init__(self, M, M_low, max_iters, max_shifts=32):
        self.M, self.M_low, self.max_iters, self.max_shifts = M, M_low, max_iters, max_shifts

    def __call__(self, xs, rhs, shifts, rsd_targets, isign=1, cb=1, rsd_low=None):
        n = len(shifts)
        if n > self.max_shifts:
            raise ValueError("too many shifts")
        xh = (C.c_void_p * n)(*[x.h.value for x in xs])
        sh = np.ascontiguousarray(shifts, dtype=np.float64)
        rs = np.ascontiguousarray(rsd_targets, dtype=np.float64)
        rl = None if rsd_low is None else np.ascontiguousarray(np.broadcast_to(rsd_low, (n,)), dtype=np.float64)
        fin = np.zeros(n)
        it, rit, corr = C.c_int(0), C.c_int(0), C.c_int(0)
        mv = C.c_ulong(0)
        check(L._lib.qphix_gpu_solve_mshift_cg_mixed(
            self.M.h, self.M_low.h, C.cast(xh, L.PP), rhs.h, n, sh.ctypes.data_as(C.c_void_p),
            rs.ctypes.data_as(C.c_void_p), None if rl is None else rl.ctypes.data_as(C.c_void_p),
            self.max_iters, isign, cb, C.byref(it), C.byref(rit), C.byref(corr),
            fin.ctypes.data_as(C.c_void_p), C.byref(mv)))
        return {"n_iters": it.value, "refine_iters": rit.value, "corrections": corr.value,
                "true_rel_resid": np.sqrt(fin), "mv_apps": mv.value}


# ---------------------------------------------------------------------------
# BLAS
# ---------------------------------------------------------------------------


def norm2(x):
    out = np.zeros(x.nrhs)
    check(L._lib.qphix_gpu_blas_norm2(x.h, out.ctypes.data_as(C.c_void_p)))
    return out


def inner_product(x, y):
    out = np.zeros(2 * x.nrhs)
    check(L._lib.qphix_gpu_blas_inner_product(x.h, y.h, out.ctypes.data_as(C.c_void_p)))
    return out[0::2] + 1j * out[1::2]


def caxpby(a, x, b, y):
    av = (C.c_double * 2)(complex(a).real, complex(a).imag)
    bv = (C.c_double * 2)(complex(b).real, complex(b).imag)
    check(L._lib.qphix_gpu_blas_caxpby(av, x.h, bv, y.h))


def caxpby_norm2(a, x, b, y):
    """y = a x + b y; returns |y|^2 per rhs (axpyNorm2)"""
    av = (C.c_double * 2)(complex(a).real, complex(a).imag)
    bv = (C.c_double * 2)(complex(b).real, complex(b).imag)
    out = np.zeros(x.nrhs)
    check(L._lib.qphix_gpu_blas_caxpby_norm2(av, x.h, bv, y.h, out.ctypes.data_as(C.c_void_p)))
    return out


def xmy_norm2(x, y, z):
    """z = x - y; returns |z|^2 per rhs (xmyNorm2Spinor; z = y: xmy2Norm2Spinor)"""
    out = np.zeros(x.nrhs)
    check(L._lib.qphix_gpu_blas_xmy_norm2(x.h, y.h, z.h, out.ctypes.data_as(C.c_void_p)))
    return out


def inner_product_norm(x, y):
    """(<x, y>, |x|^2) per rhs (innerProductNorm)"""
    out = np.zeros(3 * x.nrhs)
    check(L._lib.qphix_gpu_blas_inner_product_norm(x.h, y.h, out.ctypes.data_as(C.c_void_p)))
    return out[0::3] + 1j * out[1::3], out[2::3]


def copy(dst, src):
    check(L._lib.qphix_gpu_blas_copy(dst.h, src.h))


def zero(x):
    check(L._lib.qphix_gpu_blas_zero(x.h))


def launch_count():
    """Kernels this library has launched in the process (graph replays count
    their kernels)."""
    n = C.c_ulonglong(0)
    check(L._lib.qphix_gpu_launch_count(C.byref(n)))
    return n.value


# ---------------------------------------------------------------------------
# Dslash launch-shape autotuner
# ---------------------------------------------------------------------------
def tune_enable(enable=True):
    """Switch timing of new Dslash configurations on or off (off: default shape)."""
    lib()
    check(L._lib.qphix_gpu_tune_enable(1 if enable else 0))


def tune_entries():
    """{key: (rhs_per_thread, sites_per_thread, launch_us)} for every tuned
    Dslash configuration of this process."""
    lib()
    n = C.c_int(0)
    check(L._lib.qphix_gpu_tune_entries(C.byref(n)))
    out = {}
    buf = C.create_string_buffer(256)
    for i in range(n.value):
        r, sp, us = C.c_int(0), C.c_int(0), C.c_double(0)
        check(L._lib.qphix_gpu_tune_entry(i, buf, 256, C.byref(r), C.byref(sp), C.byref(us)))
        out[buf.value.decode()] = (r.value, sp.value, us.value)
    return out


# ---------------------------------------------------------------------------
# serving layer
# ---------------------------------------------------------------------------
OP_KINDS = {"wilson": L.WILSON, "clover": L.CLOVER_OP, "tm": L.TM, "tmclover": L.TMCLOVER}


class Server:
    """Request loop with resident ensembles (qphix_gpu_server_* in
    include/qphix_b200.h): `slots` solves in flight, each on its own stream,
    admitted against an HBM budget; results are the FP64 solutions of
    M x = b on the odd checkerboard."""

    SOLVERS = {"ru": 0, "richardson": 1}

    def __init__(self, hbm_budget_bytes, slots=4, low_prec="f16", max_bypass=4, delta=0.1, device=0,
                 solver="ru"):
        lib()
        check(L._lib.qphix_gpu_init(device))
        cfg = L.ServerConfig(int(hbm_budget_bytes), int(slots), PREC[low_prec], int(max_bypass), float(delta),
                             self.SOLVERS[solver])
        h = C.c_void_p()
        check(L._lib.qphix_gpu_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.dims = {}
        self._pending = {}  # ticket -> (rhs buffer, x buffer, request struct)

    def close(self):
        if getattr(self, "h", None):
            L._lib.qphix_gpu_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_ensemble(self, dims, gauge):
        """gauge: complex [2, 4, Vh, 3, 3] (canonical); returns the ensemble id."""
        g = np.asarray(gauge)
        g = np.ascontiguousarray(np.stack([g.real, g.imag], axis=-1), dtype=np.float64)
        arr = (C.c_int * 4)(*[int(d) for d in dims])
        eid = C.c_int(-1)
        check(L._lib.qphix_gpu_server_add_ensemble(self.h, arr, g.ctypes.data_as(C.c_void_p), C.byref(eid)))
        self.dims[eid.value] = tuple(int(d) for d in dims)
        return eid.value

    @staticmethod
    def interleave(rhs):
        """complex [(nrhs,) Vh, 4, 3] -> the C layout float64 [nrhs, Vh, 4, 3, 2]"""
        b = np.asarray(rhs)
        if b.ndim == 3:
            b = b[None]
        return np.ascontiguousarray(np.stack([b.real, b.imag], axis=-1), dtype=np.float64)

    @staticmethod
    def _request(ensemble, kind, rhs, mass, csw, mu, t_boundary, rsd_target, max_iters, out=None):
        b = np.asarray(rhs)
        if b.dtype == np.float64 and b.ndim == 5 and b.shape[-1] == 2 and b.flags.c_contiguous:
            bb = b  # already in the C layout
        else:
            bb = Server.interleave(b)
        nrhs = bb.shape[0]
        if out is None:
            xx = np.zeros_like(bb)
        else:
            if out.shape != bb.shape or out.dtype != np.float64 or not out.flags.c_contiguous:
                raise ValueError("out must be a C-contiguous float64 array shaped like the interleaved rhs")
            xx = out
        req = L.Request(int(ensemble), OP_KINDS[kind], float(mass), float(csw), float(mu), float(t_boundary),
                        int(nrhs), float(rsd_target), int(max_iters), bb.ctypes.data, xx.ctypes.data)
        return req, bb, xx

    def request_bytes(self, ensemble, kind, rhs, mass=0.0, csw=1.0, mu=0.0, t_boundary=-1.0):
        req, _, _ = self._request(ensemble, kind, rhs, mass, csw, mu, t_boundary, 1e-10, 1)
        n = C.c_size_t(0)
        check(L._lib.qphix_gpu_server_request_bytes(self.h, C.byref(req), C.byref(n)))
        return n.value

    def submit(self, ensemble, kind, rhs, mass, csw=1.0, mu=0.0, t_boundary=-1.0, rsd_target=1e-10,
               max_iters=5000, out=None):
        """rhs: complex [(nrhs,) Vh, 4, 3] odd-checkerboard spinors (or already
        interleaved, see interleave()); out: optional caller-owned float64
        buffer of the interleaved shape for the solution.  Returns a ticket;
        both buffers must stay alive until wait()."""
        req, bb, xx = self._request(ensemble, kind, rhs, mass, csw, mu, t_boundary, rsd_target, max_iters, out)
        t = C.c_longlong(0)
        check(L._lib.qphix_gpu_server_submit(self.h, C.byref(req), C.byref(t)))
        self._pending[t.value] = (bb, xx, req)
        return t.value

    def done(self, ticket):
        d = C.c_int(0)
        check(L._lib.qphix_gpu_server_poll(self.h, C.c_longlong(ticket), C.byref(d)))
        return bool(d.value)

    def wait(self, ticket, raise_on_error=True, as_complex=True):
        """(x, result dict) of a submitted request; x is complex [nrhs, Vh, 4, 3]
        (as_complex) or the interleaved float64 buffer it was written to."""
        res = L.RequestResult()
        rc = L._lib.qphix_gpu_server_wait(self.h, C.c_longlong(ticket), C.byref(res))
        bb, xx, _ = self._pending.pop(ticket)
        out = {k: getattr(res, k) for k, _ in L.RequestResult._fields_}
        if rc != L.OK:
            out["error"] = L._lib.qphix_gpu_last_error().decode()
            if raise_on_error:
                check(rc)
        return (xx[..., 0] + 1j * xx[..., 1] if as_complex else xx), out

    def stats(self):
        st = L.ServerStats()
        check(L._lib.qphix_gpu_server_get_stats(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in L.ServerStats._fields_}
