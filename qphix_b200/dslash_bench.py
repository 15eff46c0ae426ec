"""Dslash kernel micro-benchmark: one kernel variant, timed alone.

    python -m qphix_b200.dslash_bench --lattice 32 32 32 64 --prec f16 --kind clover --nrhs 1
    python -m qphix_b200.dslash_bench --lattice 16 16 16 32 --nrhs 8 --achi --norms --shape sp2

Times `--iters` launches of one Dslash variant with CUDA events on the
lattice's stream, L2 flushed (a 256 MiB write) before every launch, and
prints one JSON line: launch time and algorithmic GB/s, i.e. the compulsory
bytes per checkerboard site (each input spinor read once, output written
once, 8 links, plus the clover / full-clover term of the epilogue) times the
sites, over the launch time.  Link values do not change the timing, so a
small seeded SU(3) field is tiled over the lattice.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

BYTES = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2, "q16": 2, "q16f32": 2}
# links and clover terms, where they differ from the spinors
LINK_BYTES = {"q16f32": 4}


def algorithmic_bytes(prec, recon, kind, nrhs, achi=False):
    e = BYTES[prec]
    el = LINK_BYTES.get(prec, e)
    spinor = 24 * e + (4 if prec in ("f16", "bf16", "q16", "q16f32") else 0)
    links = 8 * recon * el
    extra = {"wilson": 0, "tm": 0, "clover": 72 * el, "tmclover": 144 * el}[kind]
    if achi and kind == "tmclover":
        extra = 72 * el
    return nrhs * (2 * spinor + (spinor if achi else 0)) + links + extra


SHAPES = {"auto": {}, "sp1": {"QPHIX_GPU_RHS_TILE": "1", "QPHIX_GPU_SITES_PER_THREAD": "1"},
          "sp2": {"QPHIX_GPU_RHS_TILE": "1", "QPHIX_GPU_SITES_PER_THREAD": "2"},
          "r2": {"QPHIX_GPU_RHS_TILE": "2", "QPHIX_GPU_SITES_PER_THREAD": "1"},
          "rhs_lanes": {"QPHIX_GPU_RHS_LANES": "1"}}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", type=int, nargs=4, default=[32, 32, 32, 64])
    ap.add_argument("--prec", default="f16", choices=list(BYTES))
    ap.add_argument("--recon", type=int, default=12, choices=[12, 18])
    ap.add_argument("--kind", default="clover", choices=["wilson", "clover", "tm", "tmclover"])
    ap.add_argument("--achi", action="store_true", help="time dslashAChiMinusBDPsi instead of dslash")
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--shape", default="auto", choices=list(SHAPES),
                    help="launch shape: auto (the autotuner's), sp1 / sp2 (sites per thread), r2 (two rhs per "
                         "thread), rhs_lanes (two rhs in the float2 lanes)")
    ap.add_argument("--norms", action="store_true",
                    help="with --achi --kind clover: fuse the |res|^2 and <res, chi> reductions (BiCGStab's "
                         "t = M s launch), folded on the device")
    args = ap.parse_args(argv)
    import os
    for k, v in SHAPES[args.shape].items():
        os.environ[k] = v

    import torch

    from . import api
    from . import fields as F

    dims = tuple(args.lattice)
    small = (8, 8, 8, 8)
    g_small = F.make_gauge(small, 5, "exp", eps=0.3)
    vh = F.vh(dims)
    reps = vh // F.vh(small)
    assert vh % F.vh(small) == 0, "lattice volume must be a multiple of 8^4"
    gauge = np.tile(g_small, (1, 1, reps, 1, 1))
    cl_small = F.make_clover(small, g_small, -0.3, 1.0)[0]
    lat = api.Lattice(dims)
    stream = torch.cuda.Stream()
    lat.set_stream(stream.cuda_stream)
    u = lat.gauge(args.prec, args.recon).upload(gauge)
    psi = lat.spinor(args.prec, args.nrhs).upload(
        np.stack([F.gaussian_spinor(dims, 3 + i) for i in range(args.nrhs)]))
    chi = lat.spinor(args.prec, args.nrhs).upload(
        np.stack([F.gaussian_spinor(dims, 30 + i) for i in range(args.nrhs)]))
    out = lat.spinor(args.prec, args.nrhs)
    clov = inv = f0 = f1 = None
    if args.kind in ("clover", "tmclover"):
        clov = lat.clover(args.prec).upload(np.tile(cl_small, (reps, 1, 1)))
        inv = lat.clover(args.prec).upload(np.tile(F.invert_clover(cl_small), (reps, 1, 1)))
    if args.kind == "tmclover":
        fi = F.twisted_full_inverse(cl_small, 0.05)
        f0 = lat.full_clover(args.prec).upload(np.tile(fi[0], (reps, 1, 1, 1)))
        f1 = lat.full_clover(args.prec).upload(np.tile(fi[1], (reps, 1, 1, 1)))
    if args.kind == "wilson":
        D = api.Dslash(lat, -1.0, 1.0, 1.0)
        run = (lambda: D.dslashAChiMinusBDPsi(out, psi, chi, u, 3.8, 0.25 / 3.8, 1, 0)) if args.achi else \
            (lambda: D.dslash(out, psi, u, 1, 0))
    elif args.kind == "tm":
        D = api.TMDslash(lat, -1.0, 1.0, 1.0, -0.2, 0.05)
        run = (lambda: D.dslashAChiMinusBDPsi(out, psi, chi, u, 3.8, 0.25, 1, 0)) if args.achi else \
            (lambda: D.dslash(out, psi, u, 1, 0))
    elif args.kind == "clover":
        D = api.ClovDslash(lat, -1.0, 1.0, 1.0)
        if args.achi and args.norms:
            run = lambda: D.dslashAChiMinusBDPsiNorms(out, psi, chi, u, clov, 0.25, 1, 0, fetch=False)
        else:
            run = (lambda: D.dslashAChiMinusBDPsi(out, psi, chi, u, clov, 0.25, 1, 0)) if args.achi else \
                (lambda: D.dslash(out, psi, u, inv, 1, 0))
    else:
        D = api.TMClovDslash(lat, -1.0, 1.0, 1.0, prec_mass_rho=0.05)
        run = (lambda: D.dslashAChiMinusBDPsi(out, psi, chi, u, clov, 0.25, 1, 0)) if args.achi else \
            (lambda: D.dslash(out, psi, u, (f0, f1), 1, 0))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    run()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.iters):
        if not args.no_flush:
            with torch.cuda.stream(stream):
                flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    t = float(np.mean(times))
    per_site = algorithmic_bytes(args.prec, args.recon, args.kind, args.nrhs, args.achi)
    gbs = per_site * vh / t / 1e9
    print(json.dumps({"lattice": list(dims), "prec": args.prec, "recon": args.recon, "kind": args.kind,
                      "achi": args.achi, "norms": args.norms, "shape": args.shape, "nrhs": args.nrhs, "sites": vh,
                      "bytes_per_site": per_site,
                      "launch_us": round(t * 1e6, 2), "min_us": round(min(times) * 1e6, 2),
                      "GBps": round(gbs, 1), "flops_per_site": args.nrhs * 1320}))


if __name__ == "__main__":
    main()
