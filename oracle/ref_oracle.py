"""ctypes front end of oracle/_ref/libqphix_ref.so -- TEST INFRASTRUCTURE ONLY.

The library holds the reference's own clover product, BLAS and Krylov solver
code (compiled from its headers by oracle/ref/Makefile); the solvers are
driven with the CPU oracle's even-odd operator as a C callback
(or_eo_apply has exactly the callback signature).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(_HERE, "_ref", "libqphix_ref.so")
_lib = None


def available():
    return os.path.exists(SO)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(SO)
        P, I_, D = C.c_void_p, C.c_int, C.c_double
        dims = C.POINTER(C.c_int)
        _lib.ref_clover_apply.argtypes = [dims, P, P, P, I_]
        _lib.ref_blas.argtypes = [dims, I_, P, P, P, P, P, P]
        _lib.ref_solve.argtypes = [dims, I_, P, P, P, P, D, I_, D, I_, I_, C.POINTER(I_), C.POINTER(D),
                                   C.POINTER(C.c_ulong)]
        _lib.ref_richardson.argtypes = [dims, P, P, P, P, D, D, I_, I_, I_, I_, C.POINTER(I_),
                                        C.POINTER(D), C.POINTER(C.c_ulong)]
        _lib.ref_minvcg.argtypes = [dims, P, P, P, P, I_, P, P, I_, I_, I_, C.POINTER(I_), P,
                                    C.POINTER(C.c_ulong)]
        for f in (_lib.ref_clover_apply, _lib.ref_blas, _lib.ref_solve, _lib.ref_richardson,
                  _lib.ref_minvcg):
            f.restype = None
    return _lib


def _dims(d):
    return (C.c_int * 4)(*d)


def _r(a):
    return O._r(a)


def clover_apply(dims, x, clov, full=False):
    xi = _r(x)
    c = _r(clov)
    out = np.empty_like(xi)
    lib().ref_clover_apply(_dims(dims), out.ctypes.data, xi.ctypes.data, c.ctypes.data, int(full))
    return O._c(out, (x.shape[0], 4, 3))


def blas(dims, op, x, y, a=(0.0, 0.0), b=(0.0, 0.0)):
    xi, yi = _r(x), _r(y).copy()
    av = np.array(a, dtype=np.float64)
    bv = np.array(b, dtype=np.float64)
    res = np.empty_like(xi)
    sc = np.zeros(2)
    lib().ref_blas(_dims(dims), op, av.ctypes.data, bv.ctypes.data, xi.ctypes.data, yi.ctypes.data,
                   res.ctypes.data, sc.ctypes.data)
    return O._c(res, (x.shape[0], 4, 3)), sc


def _apply_ptr():
    return C.cast(O.lib().or_eo_apply, C.c_void_p).value


def solve(op, kind, rhs, rsd, max_iters, omega=1.0, isign=1, cb=1):
    """kind: 'cg' | 'bicgstab' | 'mr' -- the reference solver on the oracle operator."""
    k = {"cg": 0, "bicgstab": 1, "mr": 2}[kind]
    dims = tuple(op.op.L.dims)
    x = np.zeros((op.vh, 4, 3, 2))
    b = _r(rhs)
    it = C.c_int(0)
    fin = C.c_double(0)
    mv = C.c_ulong(0)
    lib().ref_solve(_dims(dims), k, _apply_ptr(), C.cast(C.pointer(op.op), C.c_void_p), x.ctypes.data,
                    b.ctypes.data, rsd, max_iters, omega, isign, cb, C.byref(it), C.byref(fin), C.byref(mv))
    return O._c(x, (op.vh, 4, 3)), it.value, fin.value, mv.value


def richardson(op, rhs, rsd, delta, max_iters=100, inner_max=1000, isign=1, cb=1):
    dims = tuple(op.op.L.dims)
    x = np.zeros((op.vh, 4, 3, 2))
    b = _r(rhs)
    it = C.c_int(0)
    fin = C.c_double(0)
    mv = C.c_ulong(0)
    lib().ref_richardson(_dims(dims), _apply_ptr(), C.cast(C.pointer(op.op), C.c_void_p), x.ctypes.data,
                         b.ctypes.data, rsd, delta, max_iters, inner_max, isign, cb, C.byref(it),
                         C.byref(fin), C.byref(mv))
    return O._c(x, (op.vh, 4, 3)), it.value, fin.value, mv.value


def minvcg(op, rhs, shifts, rsd, max_iters=1000, isign=1, cb=1):
    dims = tuple(op.op.L.dims)
    ns = len(shifts)
    xs = [np.zeros((op.vh, 4, 3, 2)) for _ in range(ns)]
    xp = (C.c_void_p * ns)(*[x.ctypes.data for x in xs])
    sh = np.ascontiguousarray(shifts, dtype=np.float64)
    rs = np.ascontiguousarray(rsd, dtype=np.float64)
    fin = np.zeros(ns)
    it = C.c_int(0)
    mv = C.c_ulong(0)
    b = _r(rhs)
    lib().ref_minvcg(_dims(dims), _apply_ptr(), C.cast(C.pointer(op.op), C.c_void_p), C.cast(xp, C.c_void_p),
                     b.ctypes.data, ns, sh.ctypes.data, rs.ctypes.data, max_iters, isign, cb, C.byref(it),
                     fin.ctypes.data, C.byref(mv))
    return [O._c(x, (op.vh, 4, 3)) for x in xs], it.value, fin, mv.value
