"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's cpu-baseline leg as the
checker; the product never imports it.  Inputs are the canonical numpy layouts
of qphix_b200.fields (complex spinors [Vh,4,3], gauge [2,4,Vh,3,3], packed
clover [Vh,2,36], full clover [Vh,2,6,6]).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        _lib = C.CDLL(_SO)
        _declare(_lib)
    return _lib


class Lattice(C.Structure):
    _fields_ = [("dims", C.c_int * 4), ("t_boundary", C.c_double),
                ("aniso_s", C.c_double), ("aniso_t", C.c_double),
                ("use_tbc", C.c_int * 4), ("tbc", (C.c_double * 2) * 4)]


class Operator(C.Structure):
    _fields_ = [("kind", C.c_int), ("L", Lattice), ("gauge", C.c_void_p),
                ("clov", C.c_void_p), ("invclov", C.c_void_p),
                ("finv", C.c_void_p * 2), ("mass", C.c_double),
                ("twisted_mass", C.c_double), ("rho", C.c_double), ("epsilon", C.c_double)]


class SolveInfo(C.Structure):
    _fields_ = [("n_iters", C.c_int), ("rsd_sq_final", C.c_double),
                ("mv_apps", C.c_ulong), ("status", C.c_int)]


P = C.c_void_p
D = C.c_double
I_ = C.c_int


def _declare(l):
    sig = {
        "or_dslash": [C.POINTER(Lattice), P, P, P, I_, I_],
        "or_dslash_achimbdpsi": [C.POINTER(Lattice), P, P, P, P, D, D, I_, I_],
        "or_dslash_dir": [C.POINTER(Lattice), P, P, P, I_, I_],
        "or_clover_apply": [C.c_long, P, P, P],
        "or_fullclover_apply": [C.c_long, P, P, P],
        "or_clov_dslash": [C.POINTER(Lattice), P, P, P, P, I_, I_],
        "or_clov_achimbdpsi": [C.POINTER(Lattice), P, P, P, P, P, D, D, I_, I_],
        "or_tm_dslash": [C.POINTER(Lattice), P, P, P, D, D, I_, I_],
        "or_tm_achimbdpsi": [C.POINTER(Lattice), P, P, P, P, D, D, D, D, I_, I_, D],
        "or_tmclov_dslash": [C.POINTER(Lattice), P, P, P, P, P, I_, I_],
        "or_eo_apply": [C.POINTER(Operator), P, P, I_, I_],
        "or_cg": [C.POINTER(Operator), P, P, D, I_, I_, I_, C.POINTER(SolveInfo)],
        "or_cg_shift": [C.POINTER(Operator), P, P, D, D, I_, I_, I_, C.POINTER(SolveInfo)],
        "or_bicgstab": [C.POINTER(Operator), P, P, D, I_, I_, I_, C.POINTER(SolveInfo)],
        "or_mr": [C.POINTER(Operator), P, P, D, I_, D, I_, I_, C.POINTER(SolveInfo)],
        "or_minvcg": [C.POINTER(Operator), P, P, I_, P, P, I_, I_, I_,
                      C.POINTER(I_), P, C.POINTER(C.c_ulong)],
        "or_richardson_bicgstab": [C.POINTER(Operator), P, P, D, D, I_, I_, I_, I_,
                                   C.POINTER(SolveInfo)],
    }
    for name, argt in sig.items():
        f = getattr(l, name)
        f.argtypes = argt
        f.restype = None


def _r(a):
    """complex array -> contiguous float64 (re, im interleaved)."""
    a = np.asarray(a)
    if np.iscomplexobj(a):
        return np.ascontiguousarray(np.stack([a.real, a.imag], axis=-1))
    return np.ascontiguousarray(a, dtype=np.float64)


def _c(a, shape):
    a = a.reshape(shape + (2,))
    return a[..., 0] + 1j * a[..., 1]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def make_lattice(dims, t_boundary=-1.0, aniso_s=1.0, aniso_t=1.0, tbc=None):
    L = Lattice()
    for i in range(4):
        L.dims[i] = dims[i]
    L.t_boundary = t_boundary
    L.aniso_s = aniso_s
    L.aniso_t = aniso_t
    if tbc is not None:
        for i in range(4):
            if tbc[i] is not None:
                L.use_tbc[i] = 1
                L.tbc[i][0] = tbc[i].real
                L.tbc[i][1] = tbc[i].imag
    return L


class OracleOp:
    """Keeps the numpy buffers alive for an or_operator."""

    KINDS = {"wilson": 0, "clover": 1, "tm": 2, "tmclover": 3, "ndtm": 4, "ndtmclover": 5}

    def __init__(self, kind, L, gauge, clov=None, invclov=None, finv=None,
                 mass=0.0, twisted_mass=0.0, rho=0.0, epsilon=0.0):
        self.bufs = []
        op = Operator()
        op.kind = self.KINDS[kind]
        op.L = L
        g = _r(gauge)
        self.bufs.append(g)
        op.gauge = g.ctypes.data
        if clov is not None:
            c = _r(clov)
            self.bufs.append(c)
            op.clov = c.ctypes.data
        if invclov is not None:
            c = _r(invclov)
            self.bufs.append(c)
            op.invclov = c.ctypes.data
        if finv is not None:
            for i in range(2):
                c = _r(finv[i])
                self.bufs.append(c)
                op.finv[i] = c.ctypes.data
        op.mass = mass
        op.twisted_mass = twisted_mass
        op.rho = rho
        op.epsilon = epsilon
        self.op = op
        self.vh = int(np.prod(L.dims[:])) // 2
        # two-flavour operators act on [flavour][Vh][4][3]
        self.shape = (2, self.vh, 4, 3) if kind in ("ndtm", "ndtmclover") else (self.vh, 4, 3)

    def apply(self, x, isign=1, target_cb=1):
        xi = _r(x)
        out = np.empty_like(xi)
        lib().or_eo_apply(C.byref(self.op), _p(out), _p(xi), isign, target_cb)
        return _c(out, self.shape)


def dslash(L, psi, gauge, isign, cb):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, g = _r(psi), _r(gauge)
    lib().or_dslash(C.byref(L), _p(out), _p(p), _p(g), isign, cb)
    return _c(out, (psi.shape[0], 4, 3))


def dslash_achimbdpsi(L, psi, chi, gauge, alpha, beta, isign, cb):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, x, g = _r(psi), _r(chi), _r(gauge)
    lib().or_dslash_achimbdpsi(C.byref(L), _p(out), _p(p), _p(x), _p(g), alpha, beta, isign, cb)
    return _c(out, (psi.shape[0], 4, 3))


def dslash_dir(L, psi, gauge, cb, d):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, g = _r(psi), _r(gauge)
    lib().or_dslash_dir(C.byref(L), _p(out), _p(p), _p(g), cb, d)
    return _c(out, (psi.shape[0], 4, 3))


def clover_apply(x, clov):
    out = np.empty((x.shape[0], 4, 3, 2))
    xi, c = _r(x), _r(clov)
    lib().or_clover_apply(x.shape[0], _p(out), _p(xi), _p(c))
    return _c(out, (x.shape[0], 4, 3))


def fullclover_apply(x, fclov):
    out = np.empty((x.shape[0], 4, 3, 2))
    xi, c = _r(x), _r(fclov)
    lib().or_fullclover_apply(x.shape[0], _p(out), _p(xi), _p(c))
    return _c(out, (x.shape[0], 4, 3))


def clov_dslash(L, psi, gauge, invclov, isign, cb):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, g, c = _r(psi), _r(gauge), _r(invclov)
    lib().or_clov_dslash(C.byref(L), _p(out), _p(p), _p(g), _p(c), isign, cb)
    return _c(out, (psi.shape[0], 4, 3))


def clov_achimbdpsi(L, psi, chi, gauge, clov, beta, rho, isign, cb):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, x, g, c = _r(psi), _r(chi), _r(gauge), _r(clov)
    lib().or_clov_achimbdpsi(C.byref(L), _p(out), _p(p), _p(x), _p(g), _p(c), beta, rho, isign, cb)
    return _c(out, (psi.shape[0], 4, 3))


def tm_dslash(L, psi, gauge, mass, mu, isign, cb):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, g = _r(psi), _r(gauge)
    lib().or_tm_dslash(C.byref(L), _p(out), _p(p), _p(g), mass, mu, isign, cb)
    return _c(out, (psi.shape[0], 4, 3))


def tm_achimbdpsi(L, psi, chi, gauge, alpha, beta, mass, mu, isign, cb, musign=1.0):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, x, g = _r(psi), _r(chi), _r(gauge)
    lib().or_tm_achimbdpsi(C.byref(L), _p(out), _p(p), _p(x), _p(g), alpha, beta,
                           mass, mu, isign, cb, musign)
    return _c(out, (psi.shape[0], 4, 3))


def tmclov_dslash(L, psi, gauge, finv0, finv1, isign, cb):
    out = np.empty((psi.shape[0], 4, 3, 2))
    p, g, f0, f1 = _r(psi), _r(gauge), _r(finv0), _r(finv1)
    lib().or_tmclov_dslash(C.byref(L), _p(out), _p(p), _p(g), _p(f0), _p(f1), isign, cb)
    return _c(out, (psi.shape[0], 4, 3))


def _solve(fn, op, rhs, x0, *args):
    x = _r(x0 if x0 is not None else np.zeros_like(rhs)).copy()
    b = _r(rhs)
    info = SolveInfo()
    fn(C.byref(op.op), _p(x), _p(b), *args, C.byref(info))
    return _c(x, op.shape), info


def cg(op, rhs, rsd, max_iters=1000, isign=1, cb=1, x0=None):
    return _solve(lib().or_cg, op, rhs, x0, rsd, max_iters, isign, cb)


def cg_shift(op, rhs, shift, rsd, max_iters=1000, isign=1, cb=1, x0=None):
    """CG on M^+M + shift (qphix_oracle.c or_cg_shift)."""
    return _solve(lib().or_cg_shift, op, rhs, x0, shift, rsd, max_iters, isign, cb)


def bicgstab(op, rhs, rsd, max_iters=1000, isign=1, cb=1, x0=None):
    return _solve(lib().or_bicgstab, op, rhs, x0, rsd, max_iters, isign, cb)


def mr(op, rhs, rsd, max_iters=1000, omega=1.0, isign=1, cb=1, x0=None):
    return _solve(lib().or_mr, op, rhs, x0, rsd, max_iters, omega, isign, cb)


def richardson_bicgstab(op, rhs, rsd, delta, max_iters=100, inner_max_iters=1000,
                        isign=1, cb=1, x0=None):
    return _solve(lib().or_richardson_bicgstab, op, rhs, x0, rsd, delta, max_iters,
                  inner_max_iters, isign, cb)


def minvcg(op, rhs, shifts, rsd, max_iters=1000, isign=1, cb=1):
    ns = len(shifts)
    xs = [np.zeros((op.vh, 4, 3, 2)) for _ in range(ns)]
    xp = (C.c_void_p * ns)(*[x.ctypes.data for x in xs])
    sh = np.ascontiguousarray(shifts, dtype=np.float64)
    rs = np.ascontiguousarray(rsd, dtype=np.float64)
    fin = np.zeros(ns)
    n_it = I_(0)
    mv = C.c_ulong(0)
    b = _r(rhs)
    lib().or_minvcg(C.byref(op.op), C.cast(xp, C.c_void_p), _p(b), ns, _p(sh), _p(rs),
                    max_iters, isign, cb, C.byref(n_it), _p(fin), C.byref(mv))
    return [_c(x, (op.vh, 4, 3)) for x in xs], n_it.value, fin, mv.value
