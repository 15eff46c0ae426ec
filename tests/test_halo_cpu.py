"""Host side of the multi-GPU halo mode (qphix_b200/halo.py) on CPU: the
t-slab and block index arithmetic, the face order the Dslash kernel reads
against the sites the face packer writes (every ghost entry is the lattice
neighbour), and the face exchange schedule run as gloo processes (world size
2 and 3): every rank must receive its next slab's first slice and its
previous slab's last slice."""
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


GRIDS = [(2, 1, 1, 1), (1, 2, 1, 1), (1, 1, 2, 1), (1, 1, 1, 2), (1, 2, 2, 1), (2, 2, 2, 2)]


@pytest.mark.parametrize("grid", GRIDS)
def test_block_cut_covers_the_lattice(grid):
    dims = (8, 4, 4, 8)
    n = int(np.prod(grid))
    blocks = [halo.Block(dims, grid, r) for r in range(n)]
    idx = np.concatenate([b.index() for b in blocks])
    assert np.array_equal(np.sort(idx), np.arange(dims[0] * dims[1] * dims[2] * dims[3] // 2))
    psi = F.gaussian_spinor(dims, 3)
    whole = np.zeros_like(psi)
    for b in blocks:
        b.glue_spinor(whole, b.cut_spinor(psi))
        for mu in range(4):
            assert blocks[b.next[mu]].prev[mu] == b.rank
    assert np.array_equal(whole, psi)
    if grid[:3] == (1, 1, 1):  # a t cut is the t-slab decomposition
        for b in blocks:
            assert np.array_equal(b.cut_spinor(psi), halo.TSlab(dims, grid[3], b.rank).cut_spinor(psi))


def _coords(dims, s, cb):
    """local coordinates of checkerboard site s (the layout's site order)"""
    nx, ny, nz, nt = dims
    nxh = nx // 2
    xh, r = s % nxh, s // nxh
    y, r = r % ny, r // ny
    z, t = r % nz, r // nz
    return 2 * xh + ((y + z + t + cb) & 1), y, z, t


def _face_index(dims, mu, x, y, z, t):
    """the face order of the Dslash kernel's ghost reads (DslashArgs::halo)"""
    nx, ny, nz, nt = dims
    nxh = nx // 2
    return [((t * nz + z) * ny + y) >> 1, (t * nz + z) * nxh + x // 2, (t * ny + y) * nxh + x // 2,
            (z * ny + y) * nxh + x // 2][mu]


def _face_site(dims, mu, k, cb, j):
    """the packer's face site j of slice k along mu, checkerboard cb (halo.cu face_site)"""
    nx, ny, nz, nt = dims
    nxh = nx // 2
    if mu == 3:
        t, xh, r = k, j % nxh, j // nxh
        y, z = r % ny, r // ny
    elif mu == 2:
        z, xh, r = k, j % nxh, j // nxh
        y, t = r % ny, r // ny
    elif mu == 1:
        y, xh, r = k, j % nxh, j // nxh
        z, t = r % nz, r // nz
    else:
        nyh = ny // 2
        jy, r = j % nyh, j // nyh
        z, t = r % nz, r // nz
        y = 2 * jy + ((cb + k + z + t) & 1)
        xh = k >> 1
    return ((t * nz + z) * ny + y) * nxh + xh


@pytest.mark.parametrize("grid", GRIDS)
def test_block_faces_reach_the_neighbour(grid):
    """For every site on a block's last (first) slice along a cut direction,
    the ghost face entry the kernel reads is the packed site of the next
    (previous) block that is its lattice neighbour."""
    dims = (8, 4, 4, 8)
    n = int(np.prod(grid))
    blocks = [halo.Block(dims, grid, r) for r in range(n)]
    ld = blocks[0].dims
    nloc = ld[0] * ld[1] * ld[2] * ld[3] // 2
    gdims = np.array(dims)
    for b in blocks:
        for mu in range(4):
            if grid[mu] == 1:
                continue
            for cb in range(2):
                for s in range(nloc):
                    x, y, z, t = _coords(ld, s, cb)
                    c = [x, y, z, t]
                    for step, edge, nbr in ((+1, ld[mu] - 1, b.next[mu]), (-1, 0, b.prev[mu])):
                        if c[mu] != edge:
                            continue
                        j = _face_index(ld, mu, x, y, z, t)
                        # the neighbour block packs its first (last) slice of the other checkerboard
                        k = 0 if step > 0 else ld[mu] - 1
                        sn = _face_site(ld, mu, k, 1 - cb, j)
                        xn, yn, zn, tn = _coords(ld, sn, 1 - cb)
                        got = (np.array([xn, yn, zn, tn]) + np.array(blocks[nbr].origin)) % gdims
                        want = np.array(c) + np.array(b.origin)
                        want[mu] += step
                        assert np.array_equal(got, want % gdims), (b.rank, mu, cb, s, step)
                        assert 0 <= sn < nloc


def test_block_rejects_odd_extents():
    with pytest.raises(ValueError):
        halo.Block((8, 4, 4, 6), (1, 1, 1, 2), 0)  # local t extent 3
    with pytest.raises(ValueError):
        halo.Block((8, 3, 4, 8), (2, 1, 1, 1), 0)  # an x cut with an odd local Ny


def _block_rank_main(rank, world, port, grid, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = halo.Block((8, 4, 8, 8), grid, rank)
        got = {}
        for mu in range(4):  # every rank walks the cut directions in the same order
            if grid[mu] == 1:
                continue
            first = torch.full((4,), 100.0 * rank + 10 * mu + 1)
            last = torch.full((4,), 100.0 * rank + 10 * mu + 2)
            fwd, bwd = halo.exchange_faces_dir(first, last, b, mu)
            got[mu] = (float(fwd[0]), float(bwd[0]))
        out[rank] = got
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("grid", [(2, 1, 2, 1), (1, 2, 1, 2)])
def test_exchange_faces_dir_gloo(grid):
    """exchange_faces_dir on a 2 x 2 grid of blocks as four gloo processes:
    along each cut direction a rank receives its next block's first slice
    and its previous block's last slice."""
    import torch.multiprocessing as mp
    world = int(np.prod(grid))
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_block_rank_main, args=(world, port, grid, out), nprocs=world, join=True,
                           start_method="spawn")
        got = dict(out)
    for r in range(world):
        b = halo.Block((8, 4, 8, 8), grid, r)
        for mu in range(4):
            if grid[mu] == 1:
                continue
            assert got[r][mu] == (100.0 * b.next[mu] + 10 * mu + 1, 100.0 * b.prev[mu] + 10 * mu + 2), (r, mu, got)
