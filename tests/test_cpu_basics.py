"""CPU-only checks: generators, packers, the C library's exports, oracle sanity."""
import os
import re
import subprocess

import numpy as np
import pytest

from helpers import make_setup
from qphix_b200 import fields as F

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_su3_generators():
    rng = np.random.default_rng(0)
    for u in (F.random_su3_gaussian(rng, 100), F.random_su3_exp(rng, 100, 0.3),
              F.random_weak_su3(rng, 100, 0.08)):
        eye = np.einsum("nij,nkj->nik", u, np.conj(u))
        assert np.abs(eye - np.eye(3)).max() < 1e-13
        assert np.abs(np.linalg.det(u) - 1).max() < 1e-13
        # third row is conj(row0 x row1): the 12-real form reconstructs it
        assert np.abs(u[:, 2] - np.conj(np.cross(u[:, 0], u[:, 1]))).max() < 1e-13


def test_clover_hermitian_and_inverse():
    s = make_setup((4, 4, 4, 4), seed=3)
    a = F.packed_to_blocks(s["clov"][0])
    assert np.abs(a - np.conj(np.swapaxes(a, -1, -2))).max() < 1e-14
    ai = F.packed_to_blocks(s["invclov"][0])
    prod = np.einsum("...ij,...jk->...ik", ai, a)
    assert np.abs(prod - np.eye(6)).max() < 1e-12   # A^-1 A = 1 (tests-gtest/clover_product.cc:313-344)
    assert np.allclose(F.blocks_to_packed(a), s["clov"][0])


def test_unit_gauge_has_no_field_strength():
    dims = (4, 4, 4, 4)
    g = F.make_gauge(dims, 0, "unit")
    cl = F.make_clover(dims, g, 0.1, 1.0)
    assert np.allclose(cl[..., :6], 4.1) and np.allclose(cl[..., 6:], 0)


def test_qphix_packers_roundtrip():
    dims = (8, 4, 4, 4)
    lay = F.QPhiXLayout(dims, 8, 4, False, pad_xy=1, pad_xyz=2)
    x = F.gaussian_spinor(dims, 1)
    assert np.array_equal(lay.unpack_spinor(lay.pack_spinor(x)), x)
    cl = make_setup(dims)["clov"][0]
    assert np.array_equal(lay.unpack_clover(lay.pack_clover(cl)), cl)


def test_library_exports_every_header_symbol():
    from qphix_b200 import _lib
    hdr = open(os.path.join(ROOT, "include", "qphix_b200.h")).read()
    declared = set(re.findall(r"\b(qphix_gpu_\w+)\s*\(", hdr))
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.EXPORTED)


def test_dropin_headers_compile_and_link(tmp_path):
    """The drop-in headers (include/qphix/) compile as a QPhiX caller uses them
    and every C-ABI call they make resolves in the library."""
    exe = tmp_path / "dropin"
    subprocess.check_call(["g++", "-std=c++14", "-O0", "-Wall", "-Werror", "-Wno-unused-variable",
                           "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "dropin_main.cc"),
                           "-L", os.path.join(ROOT, "qphix_b200"), "-lqphix_b200", "-o", str(exe)])
    assert exe.exists()


def test_library_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from qphix_b200 import _lib
    lib = _lib.load()
    assert lib.qphix_gpu_init(0) != 0
    assert len(lib.qphix_gpu_last_error()) > 0


def test_oracle_hermiticity(oracle):
    s = make_setup((4, 4, 4, 4), seed=5)
    L = oracle.make_lattice(s["dims"], -1.0)
    x = F.gaussian_spinor(s["dims"], 1)
    y = F.gaussian_spinor(s["dims"], 2)
    a = np.vdot(y, oracle.dslash(L, x, s["gauge"], 1, 0))
    b = np.vdot(oracle.dslash(L, y, s["gauge"], -1, 1), x)
    assert abs(a - b) / abs(a) < 1e-13


def test_bench_reference_arm_runs_on_cpu():
    """`bench.py --impl reference` (QPhiX's own CPU path solving the same
    system on the host cores, else the oracle's port) prints the contract's
    line without a GPU; every step is a full solve to 1e-10."""
    import json
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "solves/s"
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_dslash
    built = ref_dslash.available("avx512") or ref_dslash.available("scalar")
    assert line["cpu_baseline"]["kind"] == ("reference" if built else "port")
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["worst_rel_resid"] <= 1e-10
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
