"""Clover term built and inverted on the device against the host
construction (clover-leaf field strength, Chroma packing) and numpy
inverses; relative tolerance 1e-13 in FP64."""
import numpy as np
import pytest

from helpers import make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("recon", [18, 12])
def test_clover_build_and_invert(recon):
    from qphix_b200 import api
    dims = (8, 4, 6, 4)
    g = F.make_gauge(dims, 17, "exp", eps=0.4)
    mass, csw, mu = -0.25, 1.3, 0.07
    ref = F.make_clover(dims, g, mass, csw)
    lat = api.Lattice(dims)
    u = lat.gauge("f64", recon).upload(g)
    for cb in (0, 1):
        A = api.clover_build(lat.clover("f64"), u, cb, mass, csw)
        got = A.download().reshape(ref[cb].shape)
        assert rel_l2(got, ref[cb]) < 1e-13, cb
        Ai = api.clover_invert(lat.clover("f64"), A)
        assert rel_l2(Ai.download().reshape(ref[cb].shape), F.invert_clover(ref[cb])) < 1e-12
        fp, fm = api.clover_invert_twisted(lat.full_clover("f64"), lat.full_clover("f64"), A, mu)
        tp, tm = F.twisted_full_inverse(ref[cb], mu)
        for fld, t in ((fp, tp), (fm, tm)):
            d = fld.download().reshape(F.vh(dims), 2, 6, 6, 2)
            assert rel_l2(d[..., 0] + 1j * d[..., 1], t) < 1e-12
        A16 = api.clover_convert(lat.clover("f16"), A)
        assert rel_l2(A16.download().reshape(ref[cb].shape), ref[cb]) < 1e-3
