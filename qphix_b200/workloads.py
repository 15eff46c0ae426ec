"""Measured runs of the solver configurations beside the headline one.

    python -m qphix_b200.workloads --config c1|c3|c4 [--reps N]

Each run builds its seeded synthetic inputs, solves through the public API
on cuda:0 and prints one JSON line (times from CUDA events on the lattice's
stream; every solution's true residual recomputed in FP64 by the library):

  c1  8^4 Wilson, Gaussian links reunitarised (18-real), kappa = 0.12, even-odd
      CG on M^+ M to 1e-10 in FP64.
  c3  24^3x48 twisted-mass clover, links exp(i 0.4 H), c_sw = 1, kappa = 0.1373,
      mu = 0.01 (QPhiX's TwistedMass / prec_mass_rho, used directly), 24
      right-hand sides in one block (12 spin-colour point sources on the
      first site of the odd checkerboard, 12 Z2 sources); BiCGStab with BF16
      storage + FP32 arithmetic iterations and FP64 reliable updates to 1e-10,
      against the plain FP64 BiCGStab one right-hand side at a time and on
      the same 24-rhs block.  The clover term is built and inverted on the
      device.
  c4  32^3x64 Wilson, links exp(i 0.3 H), kappa = 0.125, multishift CG on
      M^+ M with 16 shifts log-spaced in [1e-4, 1], one Gaussian source,
      tolerance 1e-9 per shift: the library's mixed multishift
      (MInvCGMixed: FP32 multishift, one fused, graph-captured iteration for
      all shifts, then every shift refined side by side as one 16-rhs FP32
      shifted CG on the FP64 true residuals), the same FP32 multishift with
      each shift refined on its own (FP32 single-shift corrections), and the
      FP64 multishift alone for comparison.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def _events(torch, stream):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    return e0, e1


def _setup(dims):
    import torch

    from . import api
    lat = api.Lattice(dims)
    stream = torch.cuda.Stream()
    lat.set_stream(stream.cuda_stream)
    return torch, api, lat, stream


def c1(args):
    from . import fields as F
    dims = (8, 8, 8, 8)
    kappa = 0.12
    mass = F.kappa_to_mass(kappa)
    g = F.make_gauge(dims, 101, "gaussian")
    torch, api, lat, stream = _setup(dims)
    u = lat.gauge("f64", 18).upload(g)
    M = api.EvenOddWilsonOperator(mass, u)
    b = lat.spinor("f64").upload(F.gaussian_spinor(dims, 102))
    x = lat.spinor("f64")
    cg = api.InvCG(M, 5000)
    api.zero(x)
    info = cg(x, b, 1e-10)[0]
    ts = []
    n0 = api.launch_count()
    for _ in range(args.reps):
        api.zero(x)
        e0, e1 = _events(torch, stream)
        info = cg(x, b, 1e-10)[0]
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    launches = (api.launch_count() - n0) / max(1, args.reps)
    ms = float(np.median(ts))
    return {"config": "c1", "workload": "8^4 Wilson EO, Gaussian reunitarised links 18-real, kappa 0.12, "
                                         "CG on M^+M to 1e-10, FP64",
            "solves_per_s": 1e3 / ms, "ms_per_solve": ms, "iters": info["n_iters"], "mv_apps": info["mv_apps"],
            "true_rel_resid": info["true_rel_resid"], "status": info["status"],
            # a persistent-kernel solve (small lattices, qpx_persist.cuh) is a handful of launches
            "gpu_launches_per_solve": launches}


def c3(args):
    from . import fields as F
    dims = (24, 24, 24, 48)
    kappa, mu, csw = 0.1373, 0.01, 1.0
    mass = F.kappa_to_mass(kappa)
    t0 = time.perf_counter()
    g = F.make_gauge(dims, 301, "exp", eps=0.4)
    gen_s = time.perf_counter() - t0
    torch, api, lat, stream = _setup(dims)
    u64 = lat.gauge("f64", 12).upload(g)
    ulo = lat.gauge("bf16", 12).upload(g)
    # clover term on the device: A on the odd checkerboard, (A +- i mu g5)^-1 on the even one
    a_odd = api.clover_build(lat.clover("f64"), u64, 1, mass, csw)
    a_even = api.clover_build(lat.clover("f64"), u64, 0, mass, csw)
    f0, f1 = lat.full_clover("f64"), lat.full_clover("f64")
    api.clover_invert_twisted(f0, f1, a_even, mu)
    a_lo = api.clover_convert(lat.clover("bf16"), a_odd)
    f0l = api.clover_convert(lat.full_clover("bf16"), f0)
    f1l = api.clover_convert(lat.full_clover("bf16"), f1)
    M64 = api.EvenOddTMCloverOperator(u64, a_odd, (f0, f1), prec_mass_rho=mu)
    Mlo = api.EvenOddTMCloverOperator(ulo, a_lo, (f0l, f1l), prec_mass_rho=mu)
    srcs = [F.point_source(dims, s, c) for s in range(4) for c in range(3)]
    srcs += [F.z2_noise(dims, 400 + i) for i in range(12)]
    n = len(srcs)
    b = lat.spinor("f64", n).upload(np.stack(srcs))
    x = lat.spinor("f64", n)
    ru = api.InvBiCGStabMixed(M64, Mlo, delta=0.1, max_iters=20000)
    api.zero(x)
    infos = ru(x, b, 1e-10)
    ts = []
    for _ in range(args.reps):
        api.zero(x)
        e0, e1 = _events(torch, stream)
        infos = ru(x, b, 1e-10)
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    batch_ms = float(np.median(ts))
    # the reference's own mixed-precision scheme on the same batch
    rich = api.InvRichardsonMultiPrec(M64, Mlo, "bicgstab", delta=0.005, max_iters=100, inner_max_iters=5000)
    api.zero(x)
    rinfos = rich(x, b, 1e-10)
    rts = []
    for _ in range(args.reps):
        api.zero(x)
        e0, e1 = _events(torch, stream)
        rinfos = rich(x, b, 1e-10)
        e1.record(stream)
        torch.cuda.synchronize()
        rts.append(e0.elapsed_time(e1))
    rich_ms = float(np.median(rts))
    # plain FP64 BiCGStab, one right-hand side at a time (a point and a Z2 source)
    bic = api.InvBiCGStab(M64, 20000)
    b1 = lat.spinor("f64", 1)
    x1 = lat.spinor("f64", 1)
    plain = []
    b1.upload(srcs[1])  # untimed warm-up solve: graph capture and first-launch costs
    api.zero(x1)
    bic(x1, b1, 1e-10)
    torch.cuda.synchronize()
    for k in (0, 12):
        b1.upload(srcs[k])
        api.zero(x1)
        e0, e1 = _events(torch, stream)
        inf1 = bic(x1, b1, 1e-10)[0]
        e1.record(stream)
        torch.cuda.synchronize()
        plain.append((e0.elapsed_time(e1), inf1))
    plain_ms = float(np.mean([p[0] for p in plain]))
    # plain FP64 BiCGStab on the same 24-rhs block (like for like with the
    # batched mixed solves: the block shares every link load)
    api.zero(x)
    bic(x, b, 1e-10)  # untimed warm-up: graph capture and shape tuning at 24 rhs
    api.zero(x)
    e0, e1 = _events(torch, stream)
    binfos = bic(x, b, 1e-10)
    e1.record(stream)
    torch.cuda.synchronize()
    block_ms = e0.elapsed_time(e1)
    shapes = {k: v for k, v in api.tune_entries().items() if "24x24x24x48" in k}
    return {"config": "c3", "workload": "24^3x48 TM clover EO, links exp(i 0.4 H) 12-real, csw 1.0, kappa 0.1373, "
                                         "mu 0.01, 24 rhs (12 point + 12 Z2) in one block; BiCGStab BF16 storage / "
                                         "FP32 arithmetic with FP64 reliable updates to 1e-10",
            "solves_per_s": n * 1e3 / batch_ms, "ms_per_batch": batch_ms,
            "iters": max(i["n_iters"] for i in infos), "mv_apps": infos[0]["mv_apps"],
            "worst_true_rel_resid": max(i["true_rel_resid"] for i in infos),
            "all_converged": all(i["status"] == 0 for i in infos),
            "fp64_plain": {"solves_per_s": 1e3 / plain_ms, "ms_per_solve": plain_ms,
                           "iters": [p[1]["n_iters"] for p in plain],
                           "true_rel_resid": [p[1]["true_rel_resid"] for p in plain]},
            "batched_mixed_vs_fp64_plain": (n * 1e3 / batch_ms) / (1e3 / plain_ms),
            "fp64_plain_block": {"solves_per_s": n * 1e3 / block_ms, "ms_per_batch": block_ms,
                                 "iters": max(i["n_iters"] for i in binfos),
                                 "worst_true_rel_resid": max(i["true_rel_resid"] for i in binfos),
                                 "all_converged": all(i["status"] == 0 for i in binfos)},
            "batched_mixed_vs_fp64_block": (n * 1e3 / batch_ms) / (n * 1e3 / block_ms),
            "richardson": {"delta": 0.005, "solves_per_s": n * 1e3 / rich_ms, "ms_per_batch": rich_ms,
                           "corrections": rinfos[0]["n_iters"], "mv_apps": rinfos[0]["mv_apps"],
                           "worst_true_rel_resid": max(i["true_rel_resid"] for i in rinfos),
                           "all_converged": all(i["status"] == 0 for i in rinfos),
                           "vs_fp64_plain": (n * 1e3 / rich_ms) / (1e3 / plain_ms),
                           "vs_fp64_block": block_ms / rich_ms},
            "tuned_shapes": shapes, "link_generation_s": gen_s}


def _mdagm_shift(api, M, out, x, tmp, shift):
    """out = (M^+ M + shift) x"""
    M(tmp, x, 1)
    M(out, tmp, -1)
    api.caxpby(shift, x, 1.0, out)


def c4(args):
    from . import fields as F
    dims = (32, 32, 32, 64)
    mass = F.kappa_to_mass(0.125)
    shifts = np.logspace(-4, 0, 16)
    tol = 1e-9
    t0 = time.perf_counter()
    g = F.make_gauge(dims, 501, "exp", eps=0.3)
    gen_s = time.perf_counter() - t0
    torch, api, lat, stream = _setup(dims)
    u64 = lat.gauge("f64", 12).upload(g)
    u32 = lat.gauge("f32", 12).upload(g)
    M64 = api.EvenOddWilsonOperator(mass, u64)
    M32 = api.EvenOddWilsonOperator(mass, u32)
    src = F.gaussian_spinor(dims, 502)
    b64 = lat.spinor("f64").upload(src)
    b32 = lat.spinor("f32").upload(src)
    ns = len(shifts)
    xs32 = [lat.spinor("f32") for _ in range(ns)]
    xs64 = [lat.spinor("f64") for _ in range(ns)]
    r64, t64, o64 = lat.spinor("f64"), lat.spinor("f64"), lat.spinor("f64")
    r32, d32 = lat.spinor("f32"), lat.spinor("f32")
    d64 = lat.spinor("f64")
    bnorm = float(np.sqrt(api.norm2(b64)[0]))
    ms32 = api.MInvCG(M32, 20000)
    ms64 = api.MInvCG(M64, 20000)
    one = api.MInvCG(M32, 20000, max_shifts=1)

    def true_resids(xs):
        out = []
        for k in range(ns):
            _mdagm_shift(api, M64, o64, xs[k], t64, shifts[k])
            api.copy(r64, b64)
            api.caxpby(-1.0, o64, 1.0, r64)
            out.append(float(np.sqrt(api.norm2(r64)[0])) / bnorm)
        return out

    def fp32_then_refine():
        for x in xs32:
            api.zero(x)
        it, _, mv = ms32(xs32, b32, shifts, [tol] * ns)
        corrections = 0
        for k in range(ns):
            xs64[k].convert_from(xs32[k])
            for _ in range(20):
                _mdagm_shift(api, M64, o64, xs64[k], t64, shifts[k])
                api.copy(r64, b64)
                api.caxpby(-1.0, o64, 1.0, r64)
                rn = float(np.sqrt(api.norm2(r64)[0]))
                if rn / bnorm < tol:
                    break
                r32.convert_from(r64, 1.0 / rn)
                api.zero(d32)
                # reduce the defect by what is still missing (with a margin),
                # not further: FP32 reaches ~1e-6 on its own
                need = tol * bnorm / rn
                one([d32], r32, [shifts[k]], [float(min(0.5, max(1e-5, 0.3 * need)))])
                d64.convert_from(d32, rn)
                api.caxpby(1.0, d64, 1.0, xs64[k])
                corrections += 1
        return it, mv, corrections

    fp32_then_refine()  # warm-up (graph capture, shape tuning)
    e0, e1 = _events(torch, stream)
    it32, mv32, corr = fp32_then_refine()
    e1.record(stream)
    torch.cuda.synchronize()
    per_shift_ms = e0.elapsed_time(e1)
    res_per_shift = true_resids(xs64)

    # the library's mixed multishift: FP32 multishift, then every shift
    # refined side by side as one 16-rhs shifted CG per round
    mixed = api.MInvCGMixed(M64, M32, 20000)
    rsd_low = getattr(args, "c4_rsd_low", None)
    mixed(xs64, b64, shifts, [tol] * ns, rsd_low=rsd_low)  # warm-up
    e0, e1 = _events(torch, stream)
    mo = mixed(xs64, b64, shifts, [tol] * ns, rsd_low=rsd_low)
    e1.record(stream)
    torch.cuda.synchronize()
    mixed_ms = e0.elapsed_time(e1)
    res_mixed = true_resids(xs64)
    for x in xs64:
        api.zero(x)
    ms64(xs64, b64, shifts, [tol] * ns)
    for x in xs64:
        api.zero(x)
    e0, e1 = _events(torch, stream)
    it64, _, mv64 = ms64(xs64, b64, shifts, [tol] * ns)
    e1.record(stream)
    torch.cuda.synchronize()
    fp64_ms = e0.elapsed_time(e1)
    res64 = true_resids(xs64)
    return {"config": "c4", "workload": "32^3x64 Wilson EO, links exp(i 0.3 H) 12-real, kappa 0.125, multishift CG "
                                         "on M^+M, 16 shifts logspace(1e-4, 1), tol 1e-9 per shift",
            "fp32_multishift_fp64_refined": {"ms": mixed_ms, "multishift_iters": mo["n_iters"],
                                             "refine_iters": mo["refine_iters"],
                                             "refine_rounds": mo["corrections"], "mv_apps": mo["mv_apps"],
                                             "fp32_multishift_rsd": rsd_low or tol,
                                             "worst_true_rel_resid": max(res_mixed)},
            "fp32_multishift_per_shift_refinement": {"ms": per_shift_ms, "multishift_iters": it32,
                                                     "mv_apps": mv32, "fp64_corrections": corr,
                                                     "worst_true_rel_resid": max(res_per_shift)},
            "fp64_multishift": {"ms": fp64_ms, "iters": it64, "mv_apps": mv64, "worst_true_rel_resid": max(res64)},
            "speedup_vs_fp64": fp64_ms / mixed_ms, "link_generation_s": gen_s}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", required=True, choices=["c1", "c3", "c4"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--c4-rsd-low", type=float, default=None,
                    help="c4: target of the FP32 multishift before the refinement (default: the final 1e-9)")
    args = ap.parse_args(argv)
    out = {"c1": c1, "c3": c3, "c4": c4}[args.config](args)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
