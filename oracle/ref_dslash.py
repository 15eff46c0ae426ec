"""ctypes front end of QPhiX's own code-generated Dslash family, even-odd
operators and solvers (oracle/_ref/libqphix_ref_dslash_<isa>.so, built by
oracle/ref/codegen.mk) -- TEST INFRASTRUCTURE AND CPU BASELINE ONLY.

Fields cross into the reference in its blocked host layout, packed by
qphix_b200.fields.QPhiXLayout: a reference output that matches the CPU oracle
therefore also pins that packer (transposed link storage, back links on the
other checkerboard, 12-real compression by stored columns,
qdp_packer_parscalar.h:94-129) and the oracle's Dslash family.

Two builds: "scalar" (veclen = soalen = 1, any x86-64 host) and "avx512"
(double veclen 8 with soalen 4 / 8, float veclen 16 with soalen 8; AVX-512
hosts only).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from qphix_b200 import fields as F

_HERE = os.path.dirname(os.path.abspath(__file__))
KINDS = {"wilson": 0, "clover": 1, "tm": 2, "tmclover": 3}
OPS = {"dslash": 0, "achimbdpsi": 1, "clovmult": 2, "eo": 3, "dir": 4}
SOLVERS = {"cg": 0, "bicgstab": 1}
_libs = {}


def so_path(isa):
    return os.path.join(_HERE, "_ref", f"libqphix_ref_dslash_{isa}.so")


def host_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = line.split()
                    return all(x in fl for x in ("avx512f", "avx512cd", "avx512bw", "avx512dq", "avx512vl"))
    except OSError:
        pass
    return False


def available(isa="scalar"):
    if not os.path.exists(so_path(isa)):
        return False
    return isa != "avx512" or host_has_avx512()


def lib(isa="scalar"):
    if isa not in _libs:
        if not available(isa):
            raise RuntimeError(f"reference Dslash library for {isa} is not built or not runnable here")
        l = C.CDLL(so_path(isa))
        P, I_, D = C.c_void_p, C.c_int, C.c_double
        dims = C.POINTER(C.c_int)
        l.refk_variants.argtypes = [C.POINTER(C.c_int), I_]
        l.refk_sizes.argtypes = [I_, I_, I_, I_, dims, C.POINTER(C.c_long)]
        l.refk_apply.argtypes = [I_, I_, I_, I_, dims, I_, I_, I_, P, P, P, P, P, P, P, P, P, I_, I_]
        l.refk_solve.argtypes = [I_, I_, I_, I_, dims, I_, I_, I_, P, P, P, P, P, P, P, P, D, I_, I_, I_,
                                 C.POINTER(I_), C.POINTER(D), C.POINTER(C.c_ulong), C.POINTER(D)]
        l.refk_solve_richardson.argtypes = [I_, I_, I_, dims, I_, I_, P, P, P, P, P, D, D, I_, I_, I_, I_,
                                            C.POINTER(I_), C.POINTER(D), C.POINTER(C.c_ulong), C.POINTER(D)]
        for f in (l.refk_variants, l.refk_sizes, l.refk_apply, l.refk_solve, l.refk_solve_richardson):
            f.restype = C.c_int
        _libs[isa] = l
    return _libs[isa]


def variants(isa="scalar"):
    """[(precision, veclen, soalen)] built into the library; precision 0 =
    double, 1 = float."""
    buf = (C.c_int * 30)()
    n = lib(isa).refk_variants(buf, 10)
    return [("double" if buf[3 * i] == 0 else "float", buf[3 * i + 1], buf[3 * i + 2]) for i in range(n)]


def _dims(d):
    return (C.c_int * 4)(*d)


def params(t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0, mass=0.0, mu=0.0, rho=0.0, alpha=0.0, beta=0.0,
           musign=1.0, dir=0):
    return np.array([t_boundary, aniso_s, aniso_t, mass, mu, rho, alpha, beta, musign, dir], dtype=np.float64)


class RefLattice:
    """One (precision, veclen, soalen, compress12) instance of the reference
    on one lattice, with the QPhiX-layout packers of the test suite."""

    def __init__(self, dims, prec="double", isa="scalar", veclen=None, soalen=None, compress12=False,
                 nthreads=None):
        self.isa = isa
        self.dims = tuple(dims)
        built = [v for v in variants(isa) if v[0] == prec]
        if veclen is not None:
            built = [v for v in built if v[1] == veclen]
        if soalen is not None:
            built = [v for v in built if v[2] == soalen]
        if not built:
            raise ValueError(f"no {prec} variant with veclen={veclen} soalen={soalen} in the {isa} build")
        _, self.V, self.S = built[0]
        self.prec = 0 if prec == "double" else 1
        self.dtype = np.float64 if prec == "double" else np.float32
        self.c12 = bool(compress12)
        self.nthreads = int(nthreads or os.cpu_count() or 1)
        self.layout = F.QPhiXLayout(self.dims, self.V, self.S, self.c12)
        sz = (C.c_long * 4)()
        rc = lib(isa).refk_sizes(self.prec, self.V, self.S, int(self.c12), _dims(self.dims), sz)
        if rc:
            raise RuntimeError("refk_sizes failed")
        item = np.dtype(self.dtype).itemsize
        lay = self.layout
        nc = 2 if self.c12 else 3
        mine = (lay.n_spinor_blocks * 24 * lay.S * item, lay.n_gauge_blocks * 8 * nc * 6 * lay.V * item,
                lay.n_gauge_blocks * 72 * lay.V * item, lay.n_gauge_blocks * 144 * lay.V * item)
        if tuple(sz) != mine:
            raise RuntimeError(f"layout sizes differ from Geometry's: {tuple(sz)} vs {mine}")

    # ---- packing (QPhiXLayout) -------------------------------------------
    def spinor(self, f):
        return np.ascontiguousarray(self.layout.pack_spinor(f, self.dtype))

    def gauge(self, g):
        return [np.ascontiguousarray(self.layout.pack_gauge(g, cb, self.dtype)) for cb in range(2)]

    def clover(self, c):
        return np.ascontiguousarray(self.layout.pack_clover(c, self.dtype))

    def full_clover(self, fc):
        return np.ascontiguousarray(self.layout.pack_full_clover(fc, self.dtype))

    # ---- calls -------------------------------------------------------------
    def apply(self, kind, op, psi, gauge_packed, isign=1, cb=1, chi=None, c=(None, None, None), p=None):
        """One reference call; psi / chi canonical [Vh,4,3]; gauge_packed from
        gauge(); c = the packed clover arguments of refk_apply."""
        p = params() if p is None else p
        res = np.zeros_like(self.spinor(np.zeros((F.vh(self.dims), 4, 3), complex)))
        ps = self.spinor(psi)
        ch = self.spinor(chi) if chi is not None else None
        ptr = lambda a: None if a is None else a.ctypes.data
        rc = lib(self.isa).refk_apply(self.prec, self.V, self.S, int(self.c12), _dims(self.dims), self.nthreads,
                                      KINDS[kind], OPS[op], p.ctypes.data, res.ctypes.data, ps.ctypes.data, ptr(ch),
                                      gauge_packed[0].ctypes.data, gauge_packed[1].ctypes.data, ptr(c[0]),
                                      ptr(c[1]), ptr(c[2]), isign, cb)
        if rc:
            raise RuntimeError(f"refk_apply failed ({rc})")
        return self.layout.unpack_spinor(res)

    def solve(self, kind, solver, rhs, gauge_packed, c=(None, None, None), p=None, rsd=1e-10, max_iters=5000,
              isign=1, cb=1):
        """A full reference solve (InvCG on M^dagger M or InvBiCGStab on M)
        from a zero guess.  Returns (x, n_iters, rsd_sq_final, mv_apps,
        seconds of the solver call)."""
        p = params() if p is None else p
        x = self.spinor(np.zeros((F.vh(self.dims), 4, 3), complex))
        b = self.spinor(rhs)
        it, fin, mv, sec = C.c_int(0), C.c_double(0), C.c_ulong(0), C.c_double(0)
        ptr = lambda a: None if a is None else a.ctypes.data
        rc = lib(self.isa).refk_solve(self.prec, self.V, self.S, int(self.c12), _dims(self.dims), self.nthreads,
                                      KINDS[kind], SOLVERS[solver], p.ctypes.data, gauge_packed[0].ctypes.data,
                                      gauge_packed[1].ctypes.data, ptr(c[0]), ptr(c[1]), ptr(c[2]), x.ctypes.data,
                                      b.ctypes.data, rsd, max_iters, isign, cb, C.byref(it), C.byref(fin),
                                      C.byref(mv), C.byref(sec))
        if rc:
            raise RuntimeError(f"refk_solve failed ({rc})")
        return self.layout.unpack_spinor(x), it.value, fin.value, mv.value, sec.value

    def solve_richardson(self, inner, kind, rhs, outer_fields, inner_fields, p=None, rsd=1e-10, delta=0.1,
                         max_iters=100, inner_max=5000, isign=1, cb=1):
        """InvRichardsonMultiPrec: this (double) lattice outside, `inner` (a
        float RefLattice of the same build) for the BiCGStab inside;
        *_fields = [u0, u1, c0, c1, c2] packed for each."""
        p = params() if p is None else p
        x = self.spinor(np.zeros((F.vh(self.dims), 4, 3), complex))
        b = self.spinor(rhs)
        ptrs = lambda fs: (C.c_void_p * 5)(*[None if a is None else a.ctypes.data for a in fs])
        po, pi = ptrs(outer_fields), ptrs(inner_fields)
        it, fin, mv, sec = C.c_int(0), C.c_double(0), C.c_ulong(0), C.c_double(0)
        rc = lib(self.isa).refk_solve_richardson(self.V, self.S, int(self.c12), _dims(self.dims), self.nthreads,
                                                 KINDS[kind], p.ctypes.data, C.cast(po, C.c_void_p),
                                                 C.cast(pi, C.c_void_p), x.ctypes.data, b.ctypes.data, rsd, delta,
                                                 max_iters, inner_max, isign, cb, C.byref(it), C.byref(fin),
                                                 C.byref(mv), C.byref(sec))
        if rc:
            raise RuntimeError(f"refk_solve_richardson failed ({rc})")
        return self.layout.unpack_spinor(x), it.value, fin.value, mv.value, sec.value
