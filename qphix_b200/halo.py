"""Multi-GPU halo-exchange mode: a lattice cut into slabs along t, or into
blocks along any of x, y, z, t (Block, BlockOperator, LocalBlocks below).

This replaces the face packing and exchange of the reference's multi-node path
(include/qphix/comm.h, include/qphix/face.h, and the comms split of Dyz in
include/qphix/dslash_body.h) for a t decomposition.  Each rank owns one slab
of Nt / nslabs time slices (an even number, so local and global checkerboards
agree) on its own GPU.  A Dslash on a slab reads, besides its own sites, the
neighbouring slabs' boundary time slices of the hopped field and, once per
gauge field, U_t on the previous slab's last slice.  The library packs those
faces into device buffers (qphix_gpu_halo_pack_spinor / _links) and the
halo Dslash entry points read them; moving the buffers between ranks is the
transport's job:

* `exchange_faces` with torch.distributed: batched isend / irecv (NCCL over
  NVLink between GPUs, gloo between CPU processes in the host-side tests);
* `LocalSlabs`: every slab in one process on one GPU (the neighbours' packs
  are read where they lie), which checks the halo path against the whole
  lattice.

The even-odd operators and a CG on M^+ M (`cg`, norms summed over the slabs
with a pluggable all-reduce) run distributed; the graph-captured solvers of
the library run on one GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from . import api

SIDE_FIRST, SIDE_LAST = 0, 1


class TSlab:
    """Slab `rank` of `nslabs` of a lattice cut along t."""

    def __init__(self, global_dims, nslabs, rank):
        nx, ny, nz, nt = (int(d) for d in global_dims)
        if nt % nslabs:
            raise ValueError("Nt must be divisible by the number of slabs")
        lt = nt // nslabs
        if lt % 2 or lt < 2:
            raise ValueError("each slab needs an even number (>= 2) of time slices")
        self.global_dims = (nx, ny, nz, nt)
        self.dims = (nx, ny, nz, lt)
        self.nslabs, self.rank = nslabs, rank
        self.t0 = rank * lt
        self.first, self.last = rank == 0, rank == nslabs - 1
        self.prev, self.next = (rank - 1) % nslabs, (rank + 1) % nslabs
        self.face = nx // 2 * ny * nz  # sites of one checkerboarded time slice

    # canonical arrays list checkerboard sites with t slowest, so a slab is a
    # contiguous range of them
    def _range(self):
        return slice(self.t0 * self.face, (self.t0 + self.dims[3]) * self.face)

    def cut_spinor(self, a):
        """[(nrhs,) Vh, 4, 3] of the whole lattice -> this slab's part"""
        return np.ascontiguousarray(a[..., self._range(), :, :])

    def cut_gauge(self, g):
        """[2, 4, Vh, 3, 3] -> this slab's links"""
        return np.ascontiguousarray(g[:, :, self._range()])

    def cut_clover(self, c):
        """[Vh, ...] (packed or full clover of one checkerboard) -> this slab's part"""
        return np.ascontiguousarray(c[self._range()])


def faces_struct(psi_fwd, psi_bwd, links_bwd, slab):
    f = L.HaloFaces()
    f.psi_fwd, f.psi_bwd, f.links_bwd = psi_fwd, psi_bwd, links_bwd
    f.global_first, f.global_last = int(slab.first), int(slab.last)
    return f


def _buffer(nbytes, device):
    import torch
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=device)


def exchange_faces(send_first, send_last, slab, group=None):
    """Send this slab's first slice to the previous slab and its last slice to
    the next one; return (received first slice of the next slab, received
    last slice of the previous slab).  Tag 0 carries first slices, tag 1 last
    slices, and every rank posts the same four operations in the same order,
    so the pairing holds for two slabs (where previous and next are the same
    rank) and with NCCL, which ignores tags."""
    import torch
    import torch.distributed as dist
    if slab.nslabs == 1:
        return send_first, send_last
    recv_fwd = torch.empty_like(send_first)
    recv_bwd = torch.empty_like(send_last)
    ops = [dist.P2POp(dist.isend, send_first, slab.prev, group, 0),
           dist.P2POp(dist.irecv, recv_fwd, slab.next, group, 0),
           dist.P2POp(dist.isend, send_last, slab.next, group, 1),
           dist.P2POp(dist.irecv, recv_bwd, slab.prev, group, 1)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    return recv_fwd, recv_bwd


class SlabOperator:
    """One slab's piece of an even-odd operator (include/qphix/wilson.h:49-65,
    clover.h:162-172, twisted_mass.h:62-77, twisted_mass_clover.h:92-102):
    the same two launches as the one-GPU operator, each fed the ghost faces of
    the field it hops.  `exchange(send_first, send_last) -> (fwd, bwd)` moves
    the packed faces (exchange_faces, or a LocalSlabs lookup)."""

    def __init__(self, slab, lat, p, u, exchange, clov=None, invclov=None, finv=(None, None), device="cuda:0"):
        self.slab, self.lat, self.p, self.u = slab, lat, p, u
        self.clov, self.invclov, self.finv = clov, invclov, finv
        self.exchange, self.device = exchange, device
        self.tmp = None
        nb = C.c_size_t()
        api.check(L._lib.qphix_gpu_halo_link_bytes(u.h, C.byref(nb)))
        links = _buffer(nb.value, device)
        api.check(L._lib.qphix_gpu_halo_pack_links(u.h, C.c_void_p(links.data_ptr())))
        lat.sync()
        # the previous slab's U_t, received like a last slice
        _, self.links_bwd = exchange(links, links)
        self._keep = [links]

    def pack(self, psi):
        nb = C.c_size_t()
        api.check(L._lib.qphix_gpu_halo_spinor_bytes(psi.h, C.byref(nb)))
        first, last = _buffer(nb.value, self.device), _buffer(nb.value, self.device)
        api.check(L._lib.qphix_gpu_halo_pack_spinor(psi.h, SIDE_FIRST, C.c_void_p(first.data_ptr())))
        api.check(L._lib.qphix_gpu_halo_pack_spinor(psi.h, SIDE_LAST, C.c_void_p(last.data_ptr())))
        self.lat.sync()
        return first, last

    def faces(self, psi):
        fwd, bwd = self.exchange(*self.pack(psi))
        self._keep_faces = (fwd, bwd)
        return faces_struct(fwd.data_ptr(), bwd.data_ptr(), self.links_bwd.data_ptr(), self.slab)

    def dslash(self, res, psi, isign, cb, p=None):
        """the operator kind's Dslash (with its inverse clover / twisted-mass
        epilogue) onto checkerboard cb"""
        f = self.faces(psi)
        aux, aux2 = (self.invclov, None) if self.p.kind == L.CLOVER_OP else self.finv
        api.check(L._lib.qphix_gpu_dslash_halo(C.byref(p or self.p), res.h, psi.h, self.u.h, api._h(aux),
                                               api._h(aux2), isign, cb, C.byref(f)))

    def achimbdpsi(self, res, psi, chi, alpha, beta, isign, cb, musign=1.0):
        f = self.faces(psi)
        api.check(L._lib.qphix_gpu_dslash_achimbdpsi_halo(C.byref(self.p), res.h, psi.h, chi.h, self.u.h,
                                                          api._h(self.clov), alpha, beta, isign, cb, musign,
                                                          C.byref(f)))

    def __call__(self, res, inp, isign=1, target_cb=1):
        if self.tmp is None or self.tmp.nrhs != inp.nrhs or self.tmp.prec != inp.prec:
            self.tmp = api.Field(self.lat, L.SPINOR, inp.prec, 0, inp.nrhs)
        other = 1 - target_cb
        k = self.p.kind
        self.dslash(self.tmp, inp, isign, other)
        if k == L.WILSON:
            alpha = 4.0 + self.p.mass
            self.achimbdpsi(res, self.tmp, inp, alpha, 0.25 / alpha, isign, target_cb)
        elif k == L.TM:
            self.achimbdpsi(res, self.tmp, inp, 4.0 + self.p.mass, 0.25, isign, target_cb)
        elif k in (L.CLOVER_OP, L.TMCLOVER):
            self.achimbdpsi(res, self.tmp, inp, 0.0, 0.25, isign, target_cb)
        else:
            raise ValueError("halo mode covers the Wilson, clover, twisted-mass and twisted-mass clover operators")


class LocalSlabs:
    """Every slab of a t-cut lattice in this process, on one GPU: the ghost
    faces of a slab are the neighbours' packs, read where they lie.  Used to
    check the halo path against the whole lattice."""

    def __init__(self, global_dims, nslabs, device="cuda:0"):
        self.slabs = [TSlab(global_dims, nslabs, r) for r in range(nslabs)]
        self.lats = [api.Lattice(s.dims) for s in self.slabs]
        self.device = device
        self._posted = {}

    def operators(self, make):
        """make(slab, lat, exchange) -> SlabOperator for every slab.  Each
        operator posts its link face on construction; once all exist, every
        operator takes its previous slab's."""
        def poster(r):
            def exchange(first, last):
                self._posted[r] = last
                return first, last  # replaced below, when every slab has posted
            return exchange
        ops = [make(s, lat, poster(r)) for r, (s, lat) in enumerate(zip(self.slabs, self.lats))]
        for r, op in enumerate(ops):
            op.links_bwd = self._posted[self.slabs[r].prev]
        self._posted = {}
        return ops

    def _faces(self, ops, fields):
        packs = [op.pack(x) for op, x in zip(ops, fields)]
        out = []
        for r, op in enumerate(ops):
            s = self.slabs[r]
            out.append(faces_struct(packs[s.next][0].data_ptr(), packs[s.prev][1].data_ptr(),
                                    op.links_bwd.data_ptr(), s))
        return out, packs

    def dslash(self, ops, outs, ins, isign, cb):
        """the operator kind's Dslash (with its epilogue) on every slab"""
        faces, packs = self._faces(ops, ins)
        for op, y, x, f in zip(ops, outs, ins, faces):
            aux, aux2 = (op.invclov, None) if op.p.kind == L.CLOVER_OP else op.finv
            api.check(L._lib.qphix_gpu_dslash_halo(C.byref(op.p), y.h, x.h, op.u.h, api._h(aux), api._h(aux2),
                                                   isign, cb, C.byref(f)))
        for lat in self.lats:
            lat.sync()
        del packs

    def achimbdpsi(self, ops, outs, psis, chis, alpha, beta, isign, cb, musign=1.0):
        faces, packs = self._faces(ops, psis)
        for op, y, x, c, f in zip(ops, outs, psis, chis, faces):
            api.check(L._lib.qphix_gpu_dslash_achimbdpsi_halo(C.byref(op.p), y.h, x.h, c.h, op.u.h,
                                                              api._h(op.clov), alpha, beta, isign, cb, musign,
                                                              C.byref(f)))
        for lat in self.lats:
            lat.sync()
        del packs

    def eo_apply(self, ops, outs, ins, isign=1, target_cb=1):
        """the even-odd operator on every slab (two halo launches)"""
        tmps = [api.Field(lat, L.SPINOR, x.prec, 0, x.nrhs) for lat, x in zip(self.lats, ins)]
        self.dslash(ops, tmps, ins, isign, 1 - target_cb)
        p = ops[0].p
        if p.kind == L.WILSON:
            alpha = 4.0 + p.mass
            self.achimbdpsi(ops, outs, tmps, ins, alpha, 0.25 / alpha, isign, target_cb)
        elif p.kind == L.TM:
            self.achimbdpsi(ops, outs, tmps, ins, 4.0 + p.mass, 0.25, isign, target_cb)
        else:
            self.achimbdpsi(ops, outs, tmps, ins, 0.0, 0.25, isign, target_cb)



def cg(apply, x, b, rsd_target, max_iters, allreduce=None):
    """CG on M^+ M over the slabs of a t-cut lattice, with the recurrence of
    include/qphix/invcg.h:160-340, one right-hand side per field.  x and b
    are lists of this process's slab fields (one per slab it holds);
    apply(outs, ins, isign) applies the even-odd operator on them (exchanging
    faces); allreduce(v) sums a float over the ranks (None: one process holds
    every slab, e.g. LocalSlabs).  Norms are summed over the slabs, so every
    rank takes the same steps.  Returns (iterations, |r|^2 / |b|^2)."""
    if any(f.nrhs != 1 for f in list(x) + list(b)):
        raise ValueError("the slab CG takes one right-hand side per field")
    red = allreduce or (lambda v: v)

    def fresh():
        return [api.Field(f.lat, L.SPINOR, f.prec, 0, 1) for f in x]

    r, p, mp, mmp = fresh(), fresh(), fresh(), fresh()

    def norm(fs):
        return float(red(sum(float(api.norm2(f)[0]) for f in fs)))

    bn = norm(b)
    apply(mp, x, 1)
    apply(mmp, mp, -1)
    for rr, bb, mm, pp in zip(r, b, mmp, p):
        api.copy(rr, bb)
        api.caxpby(-1.0, mm, 1.0, rr)  # r = b - M^+ M x
        api.copy(pp, rr)
    c = norm(r)
    target = rsd_target * rsd_target * bn
    it = 0
    while c > target and it < max_iters:
        apply(mp, p, 1)
        apply(mmp, mp, -1)
        a = c / norm(mp)
        for xx, rr, pp, mm in zip(x, r, p, mmp):
            api.caxpby(a, pp, 1.0, xx)
            api.caxpby(-a, mm, 1.0, rr)
        cp = norm(r)
        it += 1
        if cp <= target:
            c = cp
            break
        beta = cp / c
        for pp, rr in zip(p, r):
            api.caxpby(1.0, rr, beta, pp)  # p = r + beta p
        c = cp
    return it, c / bn if bn > 0 else 0.0


# ---------------------------------------------------------------------------
# A lattice cut along any of x, y, z, t (the 4D decomposition of
# include/qphix/comm.h:372-437): a Cartesian grid of blocks, one per rank.
# ---------------------------------------------------------------------------
class Block:
    """Block `rank` of a lattice cut into grid[0] x grid[1] x grid[2] x grid[3]
    blocks; rank = ((c_t g_z + c_z) g_y + c_y) g_x + c_x for block
    coordinates c.  Every cut direction (grid[mu] > 1) needs an even local
    extent, so block origins are even and local and global checkerboards
    agree; a cut along x also needs an even local Ny."""

    def __init__(self, global_dims, grid, rank):
        gd = tuple(int(d) for d in global_dims)
        grid = tuple(int(g) for g in grid)
        if any(d % g for d, g in zip(gd, grid)):
            raise ValueError("every global extent must be divisible by the grid")
        dims = tuple(d // g for d, g in zip(gd, grid))
        for mu in range(4):
            if grid[mu] > 1 and dims[mu] % 2:
                raise ValueError("a cut direction needs an even local extent")
        if dims[0] % 2 or (grid[0] > 1 and dims[1] % 2):
            raise ValueError("Nx must be even, and Ny too when x is cut")
        self.global_dims, self.grid, self.dims, self.rank = gd, grid, dims, rank
        c, r = [], rank
        for g in grid:
            c.append(r % g)
            r //= g
        self.coords = tuple(c)
        self.origin = tuple(ci * di for ci, di in zip(self.coords, dims))
        self.cut = sum(1 << mu for mu in range(4) if grid[mu] > 1)
        self.next = [self._rank_of(mu, +1) for mu in range(4)]
        self.prev = [self._rank_of(mu, -1) for mu in range(4)]
        self.global_first_t = self.coords[3] == 0
        self.global_last_t = self.coords[3] == grid[3] - 1

    def _rank_of(self, mu, step):
        c = list(self.coords)
        c[mu] = (c[mu] + step) % self.grid[mu]
        r = 0
        for m in (3, 2, 1, 0):
            r = r * self.grid[m] + c[m]
        return r

    def index(self):
        """the global checkerboard index of each local checkerboard site (the
        same map for both checkerboards: local and global parities agree)"""
        nx, ny, nz, nt = self.dims
        gx, gy, gz, gt = self.global_dims
        x0, y0, z0, t0 = self.origin
        nxh = nx // 2
        s = np.arange(nxh * ny * nz * nt)
        xh, r = s % nxh, s // nxh
        y, r = r % ny, r // ny
        z, t = r % nz, r // nz
        return (((t + t0) * gz + z + z0) * gy + y + y0) * (gx // 2) + x0 // 2 + xh

    def cut_spinor(self, a):
        """[(nrhs,) Vh, 4, 3] of the whole lattice (one checkerboard) -> this block's part"""
        return np.ascontiguousarray(a[..., self.index(), :, :])

    def cut_gauge(self, g):
        """[2, 4, Vh, 3, 3] -> this block's links"""
        return np.ascontiguousarray(g[:, :, self.index()])

    def cut_clover(self, c):
        """[Vh, ...] (packed or full clover of one checkerboard) -> this block's part"""
        return np.ascontiguousarray(c[self.index()])

    def glue_spinor(self, whole, part):
        """write this block's [(nrhs,) vh, 4, 3] part into the whole-lattice array"""
        whole[..., self.index(), :, :] = part


def faces4_struct(block, psi_fwd, psi_bwd, links_bwd):
    """qphix_gpu_halo_faces4 from per-direction device pointers (dicts keyed by mu)"""
    f = L.HaloFaces4()
    f.cut = block.cut
    for mu in range(4):
        if (block.cut >> mu) & 1:
            f.psi_fwd[mu], f.psi_bwd[mu], f.links_bwd[mu] = psi_fwd[mu], psi_bwd[mu], links_bwd[mu]
    f.global_first_t, f.global_last_t = int(block.global_first_t), int(block.global_last_t)
    return f


def exchange_faces_dir(send_first, send_last, block, mu, group=None):
    """exchange_faces along direction mu: this block's first slice goes to
    the previous block along mu, its last slice to the next; returns (the next
    block's first slice, the previous block's last slice).  Tags 2 mu and
    2 mu + 1; every rank exchanges the cut directions in the same order."""
    import torch
    import torch.distributed as dist
    if block.grid[mu] == 1:
        return send_first, send_last
    recv_fwd = torch.empty_like(send_first)
    recv_bwd = torch.empty_like(send_last)
    ops = [dist.P2POp(dist.isend, send_first, block.prev[mu], group, 2 * mu),
           dist.P2POp(dist.irecv, recv_fwd, block.next[mu], group, 2 * mu),
           dist.P2POp(dist.isend, send_last, block.next[mu], group, 2 * mu + 1),
           dist.P2POp(dist.irecv, recv_bwd, block.prev[mu], group, 2 * mu + 1)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    return recv_fwd, recv_bwd


class BlockOperator:
    """One block's piece of an even-odd operator for a lattice cut along any
    directions (SlabOperator's generalisation).  `exchange(mu, send_first,
    send_last) -> (fwd, bwd)` moves the packed faces along mu
    (exchange_faces_dir, or a LocalBlocks lookup)."""

    def __init__(self, block, lat, p, u, exchange, clov=None, invclov=None, finv=(None, None),
                 device="cuda:0"):
        self.block, self.lat, self.p, self.u = block, lat, p, u
        self.clov, self.invclov, self.finv = clov, invclov, finv
        self.exchange, self.device = exchange, device
        self.tmp = None
        self.links_bwd, self._keep = {}, []
        for mu in self.dirs():
            nb = C.c_size_t()
            api.check(L._lib.qphix_gpu_halo_link_bytes_dir(u.h, mu, C.byref(nb)))
            links = _buffer(nb.value, device)
            api.check(L._lib.qphix_gpu_halo_pack_links_dir(u.h, mu, C.c_void_p(links.data_ptr())))
            lat.sync()
            # the previous block's U_mu on its last slice, received like a last slice
            _, self.links_bwd[mu] = exchange(mu, links, links)
            self._keep.append(links)

    def dirs(self):
        return [mu for mu in range(4) if (self.block.cut >> mu) & 1]

    def pack(self, psi, field_cb):
        """{mu: (first, last)} slices of psi (living on checkerboard field_cb)"""
        out = {}
        for mu in self.dirs():
            nb = C.c_size_t()
            api.check(L._lib.qphix_gpu_halo_spinor_bytes_dir(psi.h, mu, C.byref(nb)))
            first, last = _buffer(nb.value, self.device), _buffer(nb.value, self.device)
            api.check(L._lib.qphix_gpu_halo_pack_spinor_dir(psi.h, mu, SIDE_FIRST, field_cb,
                                                            C.c_void_p(first.data_ptr())))
            api.check(L._lib.qphix_gpu_halo_pack_spinor_dir(psi.h, mu, SIDE_LAST, field_cb,
                                                            C.c_void_p(last.data_ptr())))
            out[mu] = (first, last)
        self.lat.sync()
        return out

    def faces(self, psi, target_cb):
        packs = self.pack(psi, 1 - target_cb)
        fwd, bwd = {}, {}
        for mu in self.dirs():
            fwd[mu], bwd[mu] = self.exchange(mu, *packs[mu])
        self._keep_faces = (fwd, bwd)
        return faces4_struct(self.block, {m: t.data_ptr() for m, t in fwd.items()},
                             {m: t.data_ptr() for m, t in bwd.items()},
                             {m: t.data_ptr() for m, t in self.links_bwd.items()})

    def dslash(self, res, psi, isign, cb):
        f = self.faces(psi, cb)
        aux, aux2 = (self.invclov, None) if self.p.kind == L.CLOVER_OP else self.finv
        api.check(L._lib.qphix_gpu_dslash_halo4(C.byref(self.p), res.h, psi.h, self.u.h, api._h(aux),
                                                api._h(aux2), isign, cb, C.byref(f)))

    def achimbdpsi(self, res, psi, chi, alpha, beta, isign, cb, musign=1.0):
        f = self.faces(psi, cb)
        api.check(L._lib.qphix_gpu_dslash_achimbdpsi_halo4(C.byref(self.p), res.h, psi.h, chi.h, self.u.h,
                                                           api._h(self.clov), alpha, beta, isign, cb, musign,
                                                           C.byref(f)))

    __call__ = SlabOperator.__call__


class LocalBlocks:
    """Every block of a cut lattice in this process, on one GPU: the ghost
    faces of a block are its neighbours' packs, read where they lie.  Checks
    the halo path against the whole lattice."""

    def __init__(self, global_dims, grid, device="cuda:0"):
        n = int(np.prod(grid))
        self.blocks = [Block(global_dims, grid, r) for r in range(n)]
        self.lats = [api.Lattice(b.dims) for b in self.blocks]
        self.device = device

    def operators(self, make):
        """make(block, lat, exchange) -> BlockOperator for every block; each
        then takes its previous blocks' link faces"""
        posted = {}

        def poster(r):
            def exchange(mu, first, last):
                posted[(r, mu)] = last
                return first, last
            return exchange
        ops = [make(b, lat, poster(r)) for r, (b, lat) in enumerate(zip(self.blocks, self.lats))]
        for r, op in enumerate(ops):
            for mu in op.dirs():
                op.links_bwd[mu] = posted[(self.blocks[r].prev[mu], mu)]
        return ops

    def _faces(self, ops, fields, target_cb):
        packs = [op.pack(x, 1 - target_cb) for op, x in zip(ops, fields)]
        out = []
        for r, op in enumerate(ops):
            b = self.blocks[r]
            fwd = {mu: packs[b.next[mu]][mu][0].data_ptr() for mu in op.dirs()}
            bwd = {mu: packs[b.prev[mu]][mu][1].data_ptr() for mu in op.dirs()}
            out.append(faces4_struct(b, fwd, bwd, {mu: t.data_ptr() for mu, t in op.links_bwd.items()}))
        return out, packs

    def dslash(self, ops, outs, ins, isign, cb):
        faces, packs = self._faces(ops, ins, cb)
        for op, y, x, f in zip(ops, outs, ins, faces):
            aux, aux2 = (op.invclov, None) if op.p.kind == L.CLOVER_OP else op.finv
            api.check(L._lib.qphix_gpu_dslash_halo4(C.byref(op.p), y.h, x.h, op.u.h, api._h(aux), api._h(aux2),
                                                    isign, cb, C.byref(f)))
        for lat in self.lats:
            lat.sync()
        del packs

    def achimbdpsi(self, ops, outs, psis, chis, alpha, beta, isign, cb, musign=1.0):
        faces, packs = self._faces(ops, psis, cb)
        for op, y, x, c, f in zip(ops, outs, psis, chis, faces):
            api.check(L._lib.qphix_gpu_dslash_achimbdpsi_halo4(C.byref(op.p), y.h, x.h, c.h, op.u.h,
                                                               api._h(op.clov), alpha, beta, isign, cb, musign,
                                                               C.byref(f)))
        for lat in self.lats:
            lat.sync()
        del packs

    eo_apply = LocalSlabs.eo_apply
