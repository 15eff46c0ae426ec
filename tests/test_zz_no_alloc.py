"""qphix_gpu_blas_norm2_noalloc against qphix_gpu_blas_norm2, through the C ABI.

The no-allocation entry point is for callers that cannot let the library
call cudaMalloc (their device memory belongs to another allocator, or an
allocation's implicit synchronisation is not acceptable where they call).
It keeps its reduction scratch in a fixed device array instead of the
lattice workspace and writes to a caller-owned device buffer; the test checks
that, on two calls in a row, it returns what the regular entry point returns
(relative 1e-13, the FP64 tolerance of the other parity tests) and what
numpy computes from the downloaded field (NUMPY_TOL), for several precisions
and right-hand-side counts; at exactly its largest size with Gaussian data
against numpy; and that
it rejects a request larger than its fixed scratch and a host result
pointer (before launching anything).  This file is collected last so a
stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# against numpy's FP64 sum of the downloaded values: FP64 fields are summed
# in FP64 throughout (1e-13); FP32-arithmetic fields sum each site's 24
# squares in FP32 before the FP64 sum over sites (about 2^-24 x 24 per site
# at worst, bounded at 1e-6)
NUMPY_TOL = {"f64": 1e-13, "f32": 1e-6, "f16": 1e-6}


def _noalloc(lib, field, out):
    import torch
    torch.cuda.synchronize()
    rc = lib.qphix_gpu_blas_norm2_noalloc(field.h, C.c_void_p(out.data_ptr()))
    return rc


@pytest.mark.parametrize("prec", ["f64", "f32", "f16"])
@pytest.mark.parametrize("nrhs", [1, 4])
def test_norm2_noalloc_matches_norm2(prec, nrhs):
    import torch

    from qphix_b200 import _lib, api
    from qphix_b200 import fields as F

    lib = _lib.load()
    dims = (8, 8, 8, 16)
    lat = api.Lattice(dims, device=0)
    x = lat.spinor(prec, nrhs).upload(np.stack([F.gaussian_spinor(dims, 70 + i) for i in range(nrhs)]))
    ref = api.norm2(x)
    xs = x.download().reshape(nrhs, -1)
    host = np.einsum("ij,ij->i", xs.conj(), xs).real  # the stored values, summed by numpy
    tol = NUMPY_TOL[prec]
    assert np.all(np.abs(ref - host) <= tol * host)
    out = torch.full((nrhs,), float("nan"), dtype=torch.float64, device="cuda:0")
    for _ in range(2):  # two calls in a row share the scratch
        out.fill_(float("nan"))
        assert _noalloc(lib, x, out) == _lib.OK, lib.qphix_gpu_last_error()
        lat.sync()
        got = out.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-13 * np.abs(ref)), (got, ref)
        assert np.all(np.abs(got - host) <= tol * host), (got, host)


def test_norm2_noalloc_rejects_oversized_request():
    import torch

    from qphix_b200 import _lib, api

    lib = _lib.load()
    lat = api.Lattice((32, 32, 32, 64), device=0)  # 8192 blocks of 128 sites
    x = lat.spinor("f16", 9)                        # 8192 * 9 > 65536 partials
    out = torch.zeros(9, dtype=torch.float64, device="cuda:0")
    assert _noalloc(lib, x, out) == _lib.EINVAL
    assert b"65536" in lib.qphix_gpu_last_error()
    x.close()
    # exactly at the limit, Gaussian data: every partial index is written
    from qphix_b200 import fields as F
    rng = np.random.default_rng(5)
    small = lat.spinor("f32", 8).upload(F.gaussian_complex(rng, (8, lat.vh, 4, 3)))
    out8 = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    for _ in range(2):
        out8.zero_()
        assert _noalloc(lib, small, out8) == _lib.OK
        lat.sync()
        xs = small.download().reshape(8, -1)
        host = np.einsum("ij,ij->i", xs.conj(), xs).real
        got = out8.cpu().numpy()
        assert np.all(np.abs(got - host) <= NUMPY_TOL["f32"] * host), (got, host)


def test_norm2_noalloc_rejects_host_result_pointer():
    from qphix_b200 import _lib, api

    lib = _lib.load()
    lat = api.Lattice((8, 8, 8, 8), device=0)
    x = lat.spinor("f64", 2)
    host = np.zeros(2)
    rc = lib.qphix_gpu_blas_norm2_noalloc(x.h, C.c_void_p(host.ctypes.data))
    assert rc == _lib.EINVAL
    assert b"device" in lib.qphix_gpu_last_error()
    assert np.all(host == 0.0)
