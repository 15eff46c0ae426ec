"""Generates tests/golden/reference_pin.npz and reference_dslash_pin.npz from
the reference's own code.

Run in a checkout that has the reference sources (oracle/ref/Makefile builds
oracle/_ref/libqphix_ref.so from them).  The fixture records, on seeded
inputs: the reference clover products (packed and full 6x6), BLAS results,
and the reference CG / BiCGStab / MR / Richardson / multishift-CG solves
driven with the oracle's even-odd clover operator.  tests/test_oracle_pin.py
checks the oracle against this file wherever the reference is absent.

reference_dslash_pin.npz holds fingerprints (norm and three seeded
projections) of the outputs of QPhiX's code-generated Dslash family and
even-odd operators (scalar build of oracle/ref/codegen.mk, 18-real links,
antiperiodic t) for every kind, call, isign and checkerboard of
tests/test_reference_dslash_pin.py.
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

DIMS = (4, 4, 4, 4)
SHIFTS = [0.01, 0.1, 0.5]


def inputs():
    from helpers import make_setup
    from qphix_b200 import fields as F
    s = make_setup(DIMS, seed=3, gauge_kind="weak", mass=0.1, mu=0.1)
    x = F.gaussian_spinor(DIMS, 1)
    y = F.gaussian_spinor(DIMS, 2)
    b = F.gaussian_spinor(DIMS, 5)
    return s, x, y, b


def main():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref")])
    import oracle as O
    import ref_oracle as R
    from qphix_b200 import fields as F
    s, x, y, b = inputs()
    out = {}
    out["clover_packed"] = R.clover_apply(DIMS, x, s["clov"][0])
    out["clover_full"] = R.clover_apply(DIMS, x, F.full_clover_to_real(s["finv"][0][0]), True)
    for op, name in [(0, "norm2"), (1, "inner")]:
        _, sc = R.blas(DIMS, op, x, y)
        out["blas_" + name] = sc
    for op, name, a, bb in [(2, "axpy", (0.3, 0.0), (0, 0)), (3, "caxpy", (0.3, -0.7), (0, 0)),
                           (5, "axpby", (0.3, 0), (-1.1, 0)), (6, "aypx", (0.45, 0), (0, 0))]:
        res, _ = R.blas(DIMS, op, x, y, a, bb)
        out["blas_" + name] = res
    res, sc = R.blas(DIMS, 4, x, y)
    out["blas_xmynorm2"] = res
    out["blas_xmynorm2_n"] = sc[0]
    L = O.make_lattice(DIMS, -1.0)
    op = O.OracleOp("clover", L, s["gauge"], clov=s["clov"][1], invclov=s["invclov"][0])
    for k in ("cg", "bicgstab", "mr"):
        xr, it, fin, mv = R.solve(op, k, b, 1e-10, 1000)
        out[f"{k}_x"], out[f"{k}_iters"], out[f"{k}_rsd"], out[f"{k}_mv"] = xr, it, fin, mv
    xr, it, fin, mv = R.richardson(op, b, 1e-10, 0.1)
    out["rich_x"], out["rich_iters"], out["rich_rsd"], out["rich_mv"] = xr, it, fin, mv
    xs, it, fin, mv = R.minvcg(op, b, SHIFTS, [1e-9] * len(SHIFTS))
    out["minv_x"], out["minv_iters"], out["minv_rsd"], out["minv_mv"] = np.stack(xs), it, fin, mv
    np.savez_compressed(os.path.join(HERE, "reference_pin.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_pin.npz"))
    dslash_fingerprints()


def dslash_fingerprints():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), "-f", "codegen.mk",
                           "ISA=scalar", "-j8"])
    import oracle as O
    import ref_dslash as R
    import test_reference_dslash_pin as T
    s, psi, chi, probes = T._golden_inputs()
    RL = R.RefLattice(T.DIMS, "double", "scalar", compress12=False, nthreads=4)
    gp = RL.gauge(s["gauge"])
    out = {}
    for name, kind, op, isign, cb in T.golden_cases():
        ref, _ = T.case(R, RL, O, s, kind, op, isign, cb, -1.0, (1.0, 1.0), psi, chi, gp)
        out[name] = T.project(ref, probes)
    np.savez_compressed(os.path.join(HERE, "reference_dslash_pin.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_dslash_pin.npz"))


if __name__ == "__main__":
    if sys.argv[1:] == ["--dslash"]:
        dslash_fingerprints()
    else:
        main()
