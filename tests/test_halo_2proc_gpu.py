"""The multi-GPU halo mode (qphix_b200/halo.py) as real processes: two gloo
ranks, each owning one t slab of an 8x4x4x16 lattice on its own lattice
object, run the SlabOperator kernels on cuda:0 and move their packed faces
through `exchange_faces` as host tensors (device -> host -> gloo -> host ->
device), and the slab-distributed CG on M^+ M (`halo.cg`, norms all-reduced
over the ranks) drives to the one-lattice solution: the glued solution
equals the oracle's CG solution to 1e-8 and its true residual is below the
target.  The same for a lattice cut along z or x into two blocks
(halo.Block / BlockOperator).  The ranks' kernels never wait on one another
(the exchange is on the host, between launches), so both can share one GPU;
on several GPUs the same code moves the faces with NCCL.
"""
import os
import socket

import numpy as np
import pytest

from helpers import make_setup, rel_l2
from qphix_b200 import fields as F

pytestmark = pytest.mark.gpu
DIMS = (8, 4, 4, 16)
ANISO = (0.9, 1.1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    from qphix_b200 import _lib as L
    from qphix_b200 import api, halo
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        s = make_setup(DIMS, seed=61, gauge_kind="weak", mass=0.1, mu=0.07)
        slab = halo.TSlab(DIMS, world, rank)
        lat = api.Lattice(slab.dims, device=0)

        def exchange(first, last):  # device packs through host tensors
            fwd, bwd = halo.exchange_faces(first.cpu(), last.cpu(), slab)
            return fwd.to("cuda:0"), bwd.to("cuda:0")

        u = lat.gauge("f64", 12).upload(slab.cut_gauge(s["gauge"]))
        A = lat.clover().upload(slab.cut_clover(s["clov"][1]))
        Ai = lat.clover().upload(slab.cut_clover(s["invclov"][0]))
        p = api.op_params(L.CLOVER_OP, -1.0, *ANISO)
        M = halo.SlabOperator(slab, lat, p, u, exchange, clov=A, invclov=Ai)
        b = F.gaussian_spinor(DIMS, 11)
        gb = lat.spinor().upload(slab.cut_spinor(b))
        gx = lat.spinor()

        def allreduce(v):
            t = torch.tensor([v], dtype=torch.float64)
            dist.all_reduce(t)
            return float(t[0])

        it, rr = halo.cg(lambda outs, ins, isign: M(outs[0], ins[0], isign, 1), [gx], [gb], 1e-10, 2000,
                         allreduce=allreduce)
        out[rank] = (it, rr, gx.download())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_process_slab_cg(oracle):
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        got = dict(out)
    its = {got[r][0] for r in range(world)}
    assert len(its) == 1, its  # every rank took the same steps
    x = np.concatenate([got[r][2] for r in range(world)])
    s = make_setup(DIMS, seed=61, gauge_kind="weak", mass=0.1, mu=0.07)
    b = F.gaussian_spinor(DIMS, 11)
    Lg = oracle.make_lattice(DIMS, -1.0, *ANISO)
    O = oracle.OracleOp("clover", Lg, s["gauge"], clov=s["clov"][1], invclov=s["invclov"][0])
    r = b - O.apply(O.apply(x, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    xo, io = oracle.cg(O, b, 1e-10, 2000)
    assert abs(its.pop() - io.n_iters) <= 1
    assert rel_l2(x, xo) < 1e-8


def _block_rank_main(rank, world, port, grid, out):
    import datetime

    import torch
    import torch.distributed as dist

    from qphix_b200 import _lib as L
    from qphix_b200 import api, halo
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        s = make_setup(BDIMS, seed=62, gauge_kind="weak", mass=0.1, mu=0.07)
        block = halo.Block(BDIMS, grid, rank)
        lat = api.Lattice(block.dims, device=0)

        def exchange(mu, first, last):  # device packs through host tensors
            fwd, bwd = halo.exchange_faces_dir(first.cpu(), last.cpu(), block, mu)
            return fwd.to("cuda:0"), bwd.to("cuda:0")

        u = lat.gauge("f64", 12).upload(block.cut_gauge(s["gauge"]))
        A = lat.clover().upload(block.cut_clover(s["clov"][1]))
        Ai = lat.clover().upload(block.cut_clover(s["invclov"][0]))
        p = api.op_params(L.CLOVER_OP, -1.0, *ANISO)
        M = halo.BlockOperator(block, lat, p, u, exchange, clov=A, invclov=Ai)
        b = F.gaussian_spinor(BDIMS, 12)
        gb = lat.spinor().upload(block.cut_spinor(b))
        gx = lat.spinor()

        def allreduce(v):
            t = torch.tensor([v], dtype=torch.float64)
            dist.all_reduce(t)
            return float(t[0])

        it, rr = halo.cg(lambda outs, ins, isign: M(outs[0], ins[0], isign, 1), [gx], [gb], 1e-10, 2000,
                         allreduce=allreduce)
        out[rank] = (it, rr, gx.download())
        dist.barrier()
    finally:
        dist.destroy_process_group()


BDIMS = (8, 4, 8, 8)


@pytest.mark.parametrize("grid", [(1, 1, 2, 1), (2, 1, 1, 1)])
def test_two_process_block_cg(oracle, grid):
    """The same as test_two_process_slab_cg for a lattice cut along z or x
    (halo.Block, BlockOperator, exchange_faces_dir)."""
    import torch.multiprocessing as mp

    from qphix_b200 import halo
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_block_rank_main, args=(world, port, grid, out), nprocs=world, join=True,
                           start_method="spawn")
        got = dict(out)
    its = {got[r][0] for r in range(world)}
    assert len(its) == 1, its
    x = np.zeros((BDIMS[0] * BDIMS[1] * BDIMS[2] * BDIMS[3] // 2, 4, 3), dtype=complex)
    for r in range(world):
        halo.Block(BDIMS, grid, r).glue_spinor(x, got[r][2])
    s = make_setup(BDIMS, seed=62, gauge_kind="weak", mass=0.1, mu=0.07)
    b = F.gaussian_spinor(BDIMS, 12)
    Lg = oracle.make_lattice(BDIMS, -1.0, *ANISO)
    O = oracle.OracleOp("clover", Lg, s["gauge"], clov=s["clov"][1], invclov=s["invclov"][0])
    r = b - O.apply(O.apply(x, 1), -1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    xo, io = oracle.cg(O, b, 1e-10, 2000)
    assert abs(its.pop() - io.n_iters) <= 1
    assert rel_l2(x, xo) < 1e-8
