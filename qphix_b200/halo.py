"""Multi-GPU halo-exchange mode: a lattice cut into slabs along t.

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
