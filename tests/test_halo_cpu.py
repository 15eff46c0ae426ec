"""Host side of the multi-GPU halo mode (qphix_b200/halo.py) on CPU: the
t-slab index arithmetic, and the face exchange schedule run as gloo
processes (world size 2 and 3): every rank must receive its next slab's
first slice and its previous slab's last slice."""
import os
import socket

import numpy as np
import pytest

from qphix_b200 import fields as F
from qphix_b200 import halo


def test_tslab_cut_covers_the_lattice():
    dims = (8, 4, 4, 16)
    psi = F.gaussian_spinor(dims, 1)
    g = F.make_gauge(dims, 2)
    cl = F.make_clover(dims, g, 0.1, 1.0)[1]
    for n in (1, 2, 4):
        slabs = [halo.TSlab(dims, n, r) for r in range(n)]
        assert all(s.dims == (8, 4, 4, 16 // n) for s in slabs)
        assert np.array_equal(np.concatenate([s.cut_spinor(psi) for s in slabs]), psi)
        assert np.array_equal(np.concatenate([s.cut_gauge(g) for s in slabs], axis=2), g)
        assert np.array_equal(np.concatenate([s.cut_clover(cl) for s in slabs]), cl)
        assert slabs[0].first and slabs[-1].last and slabs[0].prev == n - 1 and slabs[-1].next == 0
    with pytest.raises(ValueError):
        halo.TSlab(dims, 3, 0)   # 16 % 3
    with pytest.raises(ValueError):
        halo.TSlab(dims, 16, 0)  # one slice per slab


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slab = halo.TSlab((4, 4, 4, 4 * world), world, rank)
        first = torch.full((8,), 10.0 * rank + 1)   # this slab's first slice
        last = torch.full((8,), 10.0 * rank + 2)    # its last slice
        fwd, bwd = halo.exchange_faces(first, last, slab)
        out[rank] = (float(fwd[0]), float(bwd[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_faces_gloo(world):
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        got = dict(out)
    for r in range(world):
        nxt, prv = (r + 1) % world, (r - 1) % world
        assert got[r] == (10.0 * nxt + 1, 10.0 * prv + 2), (r, got)
