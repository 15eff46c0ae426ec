"""ctypes declarations of the C ABI in include/qphix_b200.h.

Loading fails loudly: there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqphix_b200.so")

OK, EINVAL, ENOMEM, ECUDA, ENOTCONV, EBREAKDOWN, EUNSUPPORTED = 0, -1, -2, -3, -4, -5, -6
F64, F32, F16, BF16, Q16, Q16F32 = 0, 1, 2, 3, 4, 5
SPINOR, GAUGE, CLOVER, FULLCLOVER = 0, 1, 2, 3
WILSON, CLOVER_OP, TM, TMCLOVER, NDTM, NDTMCLOVER = 0, 1, 2, 3, 4, 5
HOST_CANONICAL, HOST_QPHIX, HOST_QDP = 0, 1, 2
HOST_F64, HOST_F32, HOST_F16 = 0, 1, 2
SOLVER_CG, SOLVER_BICGSTAB, SOLVER_MR = 0, 1, 2


class HostLayout(C.Structure):
    _fields_ = [("kind", C.c_int), ("ft", C.c_int), ("veclen", C.c_int), ("soalen", C.c_int),
                ("compress12", C.c_int), ("pad_xy", C.c_int), ("pad_xyz", C.c_int), ("cb", C.c_int)]


class OpParams(C.Structure):
    _fields_ = [("kind", C.c_int), ("t_boundary", C.c_double), ("aniso_s", C.c_double),
                ("aniso_t", C.c_double), ("use_tbc", C.c_int * 4),
                ("tbc_phases", (C.c_double * 2) * 4), ("mass", C.c_double),
                ("twisted_mass", C.c_double), ("prec_mass_rho", C.c_double), ("epsilon", C.c_double)]


class HaloFaces(C.Structure):
    _fields_ = [("psi_fwd", C.c_void_p), ("psi_bwd", C.c_void_p), ("links_bwd", C.c_void_p),
                ("global_first", C.c_int), ("global_last", C.c_int)]


class HaloFaces4(C.Structure):
    """qphix_gpu_halo_faces4: ghost faces of a block of a lattice cut along
    any of x, y, z, t (bit mu of `cut`)"""
    _fields_ = [("cut", C.c_int), ("psi_fwd", C.c_void_p * 4), ("psi_bwd", C.c_void_p * 4),
                ("links_bwd", C.c_void_p * 4), ("global_first_t", C.c_int), ("global_last_t", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("n_iters", C.c_int), ("rsd_sq_final", C.c_double), ("site_flops", C.c_ulong),
                ("mv_apps", C.c_ulong), ("status", C.c_int), ("true_rel_resid", C.c_double),
                ("seconds", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("slots", C.c_int), ("low_prec", C.c_int),
                ("max_bypass", C.c_int), ("delta", C.c_double), ("solver", C.c_int)]


class Request(C.Structure):
    _fields_ = [("ensemble", C.c_int), ("op_kind", C.c_int), ("mass", C.c_double), ("csw", C.c_double),
                ("twisted_mass", C.c_double), ("t_boundary", C.c_double), ("nrhs", C.c_int),
                ("rsd_target", C.c_double), ("max_iters", C.c_int), ("rhs", C.c_void_p), ("x", C.c_void_p)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("n_iters", C.c_int), ("mv_apps", C.c_ulong),
                ("true_rel_resid", C.c_double), ("queue_s", C.c_double), ("solve_s", C.c_double),
                ("latency_s", C.c_double), ("bytes", C.c_size_t)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("failed", C.c_longlong), ("waiting", C.c_longlong),
                ("bypasses", C.c_longlong), ("running", C.c_int), ("running_peak", C.c_int),
                ("resident_bytes", C.c_size_t), ("reserved_bytes", C.c_size_t),
                ("reserved_peak_bytes", C.c_size_t), ("pool_used_peak_bytes", C.c_size_t)]


P = C.c_void_p
I_ = C.c_int
D = C.c_double
PP = C.POINTER(C.c_void_p)

_SIGS = {
    "qphix_gpu_version": ([], I_),
    "qphix_gpu_last_error": ([], C.c_char_p),
    "qphix_gpu_init": ([I_], I_),
    "qphix_gpu_launch_count": ([C.POINTER(C.c_ulonglong)], I_),
    "qphix_gpu_tune_enable": ([I_], I_),
    "qphix_gpu_tune_entries": ([C.POINTER(C.c_int)], I_),
    "qphix_gpu_tune_entry": ([I_, C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int),
                              C.POINTER(C.c_double)], I_),
    "qphix_gpu_lattice_create": ([C.POINTER(C.c_int), PP], I_),
    "qphix_gpu_lattice_destroy": ([P], I_),
    "qphix_gpu_lattice_set_stream": ([P, P], I_),
    "qphix_gpu_lattice_sync": ([P], I_),
    "qphix_gpu_lattice_volcb": ([P], C.c_long),
    "qphix_gpu_field_create": ([P, I_, I_, I_, I_, PP], I_),
    "qphix_gpu_field_destroy": ([P], I_),
    "qphix_gpu_field_bytes": ([P, C.POINTER(C.c_size_t)], I_),
    "qphix_gpu_field_upload": ([P, P, C.POINTER(HostLayout), I_, I_], I_),
    "qphix_gpu_field_download": ([P, P, C.POINTER(HostLayout), I_], I_),
    "qphix_gpu_field_convert": ([P, P, D], I_),
    "qphix_gpu_dslash": ([C.POINTER(OpParams), P, P, P, P, P, I_, I_], I_),
    "qphix_gpu_dslash_achimbdpsi": ([C.POINTER(OpParams), P, P, P, P, P, D, D, I_, I_, D], I_),
    "qphix_gpu_dslash_achimbdpsi_norms": ([C.POINTER(OpParams), P, P, P, P, P, D, D, I_, I_, D, P, P], I_),
    "qphix_gpu_dslash_dir": ([C.POINTER(OpParams), P, P, P, I_, I_], I_),
    "qphix_gpu_halo_spinor_bytes": ([P, C.POINTER(C.c_size_t)], I_),
    "qphix_gpu_halo_pack_spinor": ([P, I_, P], I_),
    "qphix_gpu_halo_link_bytes": ([P, C.POINTER(C.c_size_t)], I_),
    "qphix_gpu_halo_pack_links": ([P, P], I_),
    "qphix_gpu_dslash_halo": ([C.POINTER(OpParams), P, P, P, P, P, I_, I_, C.POINTER(HaloFaces)], I_),
    "qphix_gpu_dslash_achimbdpsi_halo": ([C.POINTER(OpParams), P, P, P, P, P, D, D, I_, I_, D,
                                          C.POINTER(HaloFaces)], I_),
    "qphix_gpu_halo_face_sites": ([P, I_, C.POINTER(C.c_size_t)], I_),
    "qphix_gpu_halo_spinor_bytes_dir": ([P, I_, C.POINTER(C.c_size_t)], I_),
    "qphix_gpu_halo_pack_spinor_dir": ([P, I_, I_, I_, P], I_),
    "qphix_gpu_halo_link_bytes_dir": ([P, I_, C.POINTER(C.c_size_t)], I_),
    "qphix_gpu_halo_pack_links_dir": ([P, I_, P], I_),
    "qphix_gpu_dslash_halo4": ([C.POINTER(OpParams), P, P, P, P, P, I_, I_, C.POINTER(HaloFaces4)], I_),
    "qphix_gpu_dslash_achimbdpsi_halo4": ([C.POINTER(OpParams), P, P, P, P, P, D, D, I_, I_, D,
                                           C.POINTER(HaloFaces4)], I_),
    "qphix_gpu_dslash_two_flav_clover": ([C.POINTER(OpParams), P, P, P, P, P, P, I_, I_], I_),
    "qphix_gpu_clover_apply": ([P, P, P], I_),
    "qphix_gpu_clover_build": ([P, P, I_, D, D, D], I_),
    "qphix_gpu_clover_invert": ([P, P], I_),
    "qphix_gpu_clover_invert_twisted": ([P, P, P, D], I_),
    "qphix_gpu_clover_invert_ndtm": ([P, P, P, P, D, D], I_),
    "qphix_gpu_two_flav_clover_apply": ([P, P, P, P, P, I_], I_),
    "qphix_gpu_clover_convert": ([P, P], I_),
    "qphix_gpu_eo_op_create": ([C.POINTER(OpParams), P, P, P, P, P, PP], I_),
    "qphix_gpu_eo_op_destroy": ([P], I_),
    "qphix_gpu_eo_op_apply": ([P, P, P, I_, I_], I_),
    "qphix_gpu_solve_cg": ([P, P, P, D, I_, I_, I_, C.POINTER(SolveInfo)], I_),
    "qphix_gpu_solve_bicgstab": ([P, P, P, D, I_, I_, I_, C.POINTER(SolveInfo)], I_),
    "qphix_gpu_solve_mr": ([P, P, P, D, I_, D, I_, I_, C.POINTER(SolveInfo)], I_),
    "qphix_gpu_solve_mr_smoother": ([P, P, P, I_, D, I_, I_, C.POINTER(SolveInfo)], I_),
    "qphix_gpu_solve_mshift_cg": ([P, PP, P, I_, P, P, I_, I_, I_, C.POINTER(C.c_int), P,
                                   C.POINTER(C.c_ulong)], I_),
    "qphix_gpu_solve_bicgstab_mixed": ([P, P, P, P, D, D, I_, I_, I_, C.POINTER(SolveInfo)], I_),
    "qphix_gpu_solve_richardson": ([P, P, I_, P, P, D, D, I_, I_, I_, I_, C.POINTER(SolveInfo)], I_),
    "qphix_gpu_solve_cg_shifted": ([P, P, P, P, P, I_, I_, I_, C.POINTER(SolveInfo)], I_),
    "qphix_gpu_solve_mshift_cg_mixed": ([P, P, PP, P, I_, P, P, P, I_, I_, I_, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int), C.POINTER(C.c_int), P, C.POINTER(C.c_ulong)], I_),
    "qphix_gpu_blas_norm2": ([P, P], I_),
    "qphix_gpu_blas_norm2_noalloc": ([P, P], I_),
    "qphix_gpu_blas_inner_product": ([P, P, P], I_),
    "qphix_gpu_blas_caxpby": ([P, P, P, P], I_),
    "qphix_gpu_blas_caxpby_norm2": ([P, P, P, P, P], I_),
    "qphix_gpu_blas_xmy_norm2": ([P, P, P, P], I_),
    "qphix_gpu_blas_inner_product_norm": ([P, P, P], I_),
    "qphix_gpu_blas_copy": ([P, P], I_),
    "qphix_gpu_blas_zero": ([P], I_),
    "qphix_gpu_server_create": ([C.POINTER(ServerConfig), PP], I_),
    "qphix_gpu_server_add_ensemble": ([P, C.POINTER(C.c_int), P, C.POINTER(C.c_int)], I_),
    "qphix_gpu_server_request_bytes": ([P, C.POINTER(Request), C.POINTER(C.c_size_t)], I_),
    "qphix_gpu_server_submit": ([P, C.POINTER(Request), C.POINTER(C.c_longlong)], I_),
    "qphix_gpu_server_poll": ([P, C.c_longlong, C.POINTER(C.c_int)], I_),
    "qphix_gpu_server_wait": ([P, C.c_longlong, C.POINTER(RequestResult)], I_),
    "qphix_gpu_server_get_stats": ([P, C.POINTER(ServerStats)], I_),
    "qphix_gpu_server_destroy": ([P], I_),
}

EXPORTED = sorted(_SIGS)

_lib = None


class QPhiXGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load(path: str | None = None):
    """Load (once) and return the C library; raises if it is missing.
    QPHIX_B200_LIBRARY names another build of it (e.g. a variant with other
    kernel register budgets) to load instead of the in-tree one."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("QPHIX_B200_LIBRARY") or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m qphix_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (argt, rest) in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = argt
        f.restype = rest
    _lib = lib
    return lib


def check(rc):
    if rc != OK:
        msg = _lib.qphix_gpu_last_error().decode() if _lib else "library not loaded"
        raise QPhiXGPUError(rc, msg)
    return rc
