"""Shared fixtures for the parity tests: seeded fields and comparison helpers."""
import numpy as np

from qphix_b200 import fields as F


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_setup(dims, seed=11, gauge_kind="gaussian", mass=0.1, csw=1.0, mu=0.05):
    g = F.make_gauge(dims, seed, gauge_kind)
    cl = F.make_clover(dims, g, mass, csw)          # [2 cb, Vh, 2, 36]
    inv = np.stack([F.invert_clover(cl[0]), F.invert_clover(cl[1])])
    finv = [F.twisted_full_inverse(cl[cb], mu) for cb in range(2)]  # [cb][+/-]
    return dict(dims=dims, gauge=g, clov=cl, invclov=inv, finv=finv, mass=mass, mu=mu)


TOL = {"f64": 1e-13, "f32": 1e-6, "f16": 4e-3, "bf16": 3e-2, "q16": 1e-3, "q16f32": 1e-4}
