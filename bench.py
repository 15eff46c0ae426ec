#!/usr/bin/env python
"""Headline benchmark: clover solves/s to a 1e-10 FP64 true residual.

Workload (one step = one batched solve): even-odd preconditioned Wilson-clover
operator on a 16^3x32 lattice, kappa = 0.1360 (bare mass 1/(2 kappa) - 4),
c_sw = 1.0, links exp(i 0.3 H) with H drawn from the Gaussian unitary
ensemble (stored 12-real), antiperiodic in t.  `--batch` right-hand sides are
solved together to a 1e-10 relative true (FP64) residual by QPhiX's
mixed-precision scheme, InvRichardsonMultiPrec: FP64 outer defect correction
(solution and true residual in FP64), inner BiCGStab on FP16-storage /
FP32-arithmetic fields reducing each correction's residual by delta = 0.005.
`--solver ru` selects BiCGStab with reliable updates (delta 0.03) instead;
the other solver, and the default solver with a Q16 inner operator, are timed
beside it.  Plain FP64 BiCGStab is timed on the same 8-rhs block (the ratio's
denominator) and on one rhs at a time.

value  = solves/s with the right-hand sides resident in HBM
e2e    = solves/s through the C ABI with host buffers: pinned host -> device
         upload of the sources, solve, device -> host download of x per step
roofline: the dominant kernel (the FP16 clover Dslash A chi - b D psi of the
         inner solve), timed alone on the same lattice with L2 flushed before
         every launch; the operator's first kernel (A^-1 D psi) beside it.
cpu_baseline: QPhiX's own CPU path (its code-generated AVX-512 kernels and
         InvRichardsonMultiPrec / InvBiCGStab, built from the reference
         sources) solving one right-hand side of the same system to 1e-10 on
         all host cores; --impl reference times the same solves per step.

At N = 1 the other configurations follow the headline (extra_configs():
8^4 CG, 24^3x48 24-rhs TM clover, 32^3x64 16-shift multishift, and the
2000-request serving stream whose latency p50 / p99 is the metric's "p99
ms"); --no-extra skips them.

N > 1 GPUs: independent replicas (the path does not shard across GPUs here);
value = all ranks' solves / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

KAPPA = 0.1360
CSW = 1.0
EPS = 0.3
DIMS = (16, 16, 16, 32)
RSD = 1e-10
# measured on this workload (8 rhs, FP16 inner): Richardson 0.003-0.01 all
# reach 1e-10 in 6 corrections, 0.005 with the fewest inner iterations;
# reliable-update BiCGStab is fastest at 0.03
DEFAULT_DELTA = {"richardson": 0.005, "ru": 0.03}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--inner", default="f16", choices=["f16", "bf16", "q16", "q16f32", "f32"])
    ap.add_argument("--inner-recon", type=int, default=12, choices=[12, 18],
                    help="link storage of the inner operator (12- or 18-real)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other configurations (8^4 CG, 24^3x48 24-rhs TM clover, 32^3x64 16-shift "
                         "multishift, the 2000-request serving stream) measured after the headline at N = 1")
    ap.add_argument("--solver", default="richardson", choices=["ru", "richardson"],
                    help="ru: BiCGStab with reliable updates; richardson: InvRichardsonMultiPrec")
    ap.add_argument("--delta", type=float, default=None,
                    help="residual reduction per correction / reliable update (default: richardson "
                         f"{DEFAULT_DELTA['richardson']}, ru {DEFAULT_DELTA['ru']})")
    args = ap.parse_args()
    if args.delta is None:
        args.delta = DEFAULT_DELTA[args.solver]
    return args


# ---------------------------------------------------------------------------
def make_inputs(dims, batch, seed=2024):
    from qphix_b200 import fields as F
    g = F.make_gauge(dims, seed, "exp", eps=EPS)
    mass = F.kappa_to_mass(KAPPA)
    cl = F.make_clover(dims, g, mass, CSW)
    inv_even = F.invert_clover(cl[0])
    rhs = np.stack([F.gaussian_spinor(dims, seed + 100 + i) for i in range(batch)])
    return dict(gauge=g, clov_odd=cl[1], invclov_even=inv_even, rhs=rhs, mass=mass)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """Per-site DRAM traffic of the profiled kernels (profiles/traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ---------------------------------------------------------------------------
REF_DELTA = 0.01  # the reference's fastest Richardson delta on this workload


class ReferenceCPU:
    """QPhiX's own CPU implementation of the path on the host cores: its
    code-generated AVX-512 (else scalar) Dslash kernels behind its
    EvenOddCloverOperator, InvBiCGStab and InvRichardsonMultiPrec templates,
    compiled from the reference sources (oracle/_ref, oracle/ref/codegen.mk).
    Without that build, the CPU oracle's port of the same solver stands in
    (kind "port")."""

    def __init__(self, inputs, dims):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        self.inputs, self.dims = inputs, dims
        self.cores = os.cpu_count() or 1
        self.model = _cpu_model()
        import ref_dslash as R
        self.isa = "avx512" if R.available("avx512") else ("scalar" if R.available("scalar") else None)
        if self.isa is None:
            self.kind = "port"
            return
        self.kind = "reference"
        self.R = R
        vo, so, vi, si = (8, 8, 16, 8) if self.isa == "avx512" else (1, 1, 1, 1)
        self.layouts = f"double V={vo} S={so}, float V={vi} S={si}, 12-real links"
        self.outer = R.RefLattice(dims, "double", self.isa, vo, so, True, self.cores)
        self.inner = R.RefLattice(dims, "float", self.isa, vi, si, True, self.cores)
        self.fo = self._fields(self.outer)
        self.fi = self._fields(self.inner)
        self.p = R.params(t_boundary=-1.0)

    def _fields(self, RL):
        g = RL.gauge(self.inputs["gauge"])
        return [g[0], g[1], RL.clover(self.inputs["clov_odd"]), RL.clover(self.inputs["invclov_even"]), None]

    def mixed(self, rhs):
        """one full InvRichardsonMultiPrec<double, float> solve to 1e-10:
        (seconds, outer iterations, relative residual, operator applications)"""
        if self.kind == "port":
            return self.fp64(rhs)
        x, it, fin, mv, sec = self.outer.solve_richardson(self.inner, "clover", rhs, self.fo, self.fi, p=self.p,
                                                          rsd=RSD, delta=REF_DELTA, max_iters=100,
                                                          inner_max=5000)
        return sec, it, float(np.sqrt(max(fin, 0.0))), mv

    def fp64(self, rhs):
        """one full FP64 InvBiCGStab solve to 1e-10 (same tuple)"""
        if self.kind == "port":
            import oracle as O
            L = O.make_lattice(self.dims, -1.0)
            op = O.OracleOp("clover", L, self.inputs["gauge"], clov=self.inputs["clov_odd"],
                            invclov=self.inputs["invclov_even"])
            t0 = time.perf_counter()
            _, info = O.bicgstab(op, rhs, RSD, 5000)
            sec = time.perf_counter() - t0
            return sec, info.n_iters, float(np.sqrt(max(info.rsd_sq_final, 0.0)) / np.linalg.norm(rhs)), \
                info.mv_apps
        c = self.fo
        x, it, fin, mv, sec = self.outer.solve("clover", "bicgstab", rhs, c[:2], c=(c[2], c[3], None), p=self.p,
                                               rsd=RSD, max_iters=5000)
        return sec, it, float(np.sqrt(max(fin, 0.0)) / np.linalg.norm(rhs)), mv

    def describe(self, what):
        if self.kind == "port":
            return (f"{what} by the CPU oracle's port of include/qphix/invbicgstab.h (the reference's own "
                    f"build is absent), {self.cores} OpenMP threads, {self.model}")
        return (f"{what}: QPhiX's own code-generated {self.isa} kernels and solver templates "
                f"({self.layouts}), {self.cores} OpenMP threads, {self.model}")


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def cpu_baseline_leg(inputs, dims, repeats=2):
    """The bench line's cpu_baseline: full single-rhs solves of the headline
    system by the reference on the host cores (mixed precision, its
    InvRichardsonMultiPrec, is the value; FP64 InvBiCGStab beside it)."""
    ref = ReferenceCPU(inputs, dims)
    rhs = inputs["rhs"][0]
    ref.mixed(rhs)  # first call: page-in and thread start-up
    runs = [ref.mixed(rhs) for _ in range(repeats)]
    sec = statistics.median(r[0] for r in runs)
    f64 = ref.fp64(rhs)
    what = (f"{repeats} full InvRichardsonMultiPrec<double, float> solves (inner BiCGStab, delta {REF_DELTA}) of "
            f"one rhs of the headline system to 1e-10 (median)") if ref.kind == "reference" else \
        f"{repeats} full FP64 BiCGStab solves of one rhs to 1e-10 (median)"
    return {"value": 1.0 / sec, "unit": "solves/s", "cores": ref.cores, "kind": ref.kind,
            "sample": ref.describe(what), "isa": ref.isa,
            "mixed": {"seconds": sec, "outer_iters": runs[-1][1], "rel_resid": runs[-1][2], "mv_apps": runs[-1][3]},
            "fp64_bicgstab": {"solves_per_s": 1.0 / f64[0], "iters": f64[1], "rel_resid": f64[2],
                              "mv_apps": f64[3]}}


def run_reference(args, rank, world):
    """--impl reference: QPhiX's own CPU implementation of the path on the
    host cores (rank 0 only).  One step = one full solve to 1e-10 of one of
    the headline system's right-hand sides (the reference has no multi-rhs
    solver) with its mixed-precision InvRichardsonMultiPrec<double, float>;
    value = solves / summed solver time."""
    if rank != 0:
        return
    inputs = make_inputs(DIMS, args.batch)
    ref = ReferenceCPU(inputs, DIMS)
    for i in range(args.warmup):
        ref.mixed(inputs["rhs"][i % args.batch])
    runs = [ref.mixed(inputs["rhs"][i % args.batch]) for i in range(args.steps)]
    total = sum(r[0] for r in runs)
    v = args.steps / total
    f64 = ref.fp64(inputs["rhs"][0])
    what = (f"each step one full InvRichardsonMultiPrec<double, float> solve (inner BiCGStab, delta {REF_DELTA}) "
            f"of one rhs to 1e-10" if ref.kind == "reference" else "each step one full FP64 BiCGStab solve")
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total * 1e3 / args.steps, 3),
            "higher_is_better": True, "data": "synthetic (seeded)",
            "config": config_dict(args.batch, args.inner, args.solver, args.inner_recon, args.delta),
            "reference_path": ref.describe(what),
            "worst_rel_resid": max(r[2] for r in runs), "outer_iters": runs[-1][1], "mv_apps": runs[-1][3],
            "fp64_bicgstab": {"solves_per_s": round(1.0 / f64[0], 4), "iters": f64[1], "rel_resid": f64[2]},
            "cpu_baseline": {"value": round(v, 4), "unit": "solves/s", "cores": ref.cores, "kind": ref.kind,
                             "sample": ref.describe(what)},
            "e2e": {"value": round(v, 4), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def extra_configs():
    """The benchmark's other configurations, each measured once after the
    headline (N = 1, rank 0): 8^4 Wilson CG, the 24^3x48 24-rhs batched
    twisted-mass clover solve, the 32^3x64 16-shift multishift CG
    (qphix_b200.workloads) and the 2000-request Poisson serving stream at 70 %
    of measured capacity (qphix_b200.serve_bench, requests solved with
    reliable-update BiCGStab: on the four-volume mix it gave the lower p99
    latency; InvRichardsonMultiPrec the higher capacity, with a longer
    tail), whose latency p50 / p99 are the metric's "p99 ms"."""
    import types

    from qphix_b200 import serve_bench, workloads
    out = {}
    for name, fn in (("c1", workloads.c1), ("c3", workloads.c3), ("c4", workloads.c4)):
        t0 = time.perf_counter()
        try:
            out[name] = fn(types.SimpleNamespace(reps=2))
        except Exception as e:  # pragma: no cover - reported, the headline still prints
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = round(time.perf_counter() - t0, 1)
    t0 = time.perf_counter()
    try:
        out["serve"] = serve_bench.run(["--requests", "2000", "--load", "0.7", "--solver", "ru"])
    except Exception as e:  # pragma: no cover
        out["serve"] = {"error": f"{type(e).__name__}: {e}"}
    out["serve"]["wall_s_total"] = round(time.perf_counter() - t0, 1)
    return out


METRIC = "Clover solves/s @1e-10 mixed vs FP64 plain, 1 B200; Dslash HBM GB/s; p99 ms"


def config_dict(batch, inner, solver="richardson", inner_recon=12, delta=None):
    how = ("BiCGStab with reliable updates (FP64 true residual / solution, iterations in "
           f"{inner} storage ({inner_recon}-real links) + FP32 arithmetic, delta {delta})" if solver == "ru" else
           f"InvRichardsonMultiPrec (FP64 outer defect correction, BiCGStab inner in {inner} storage "
           f"({inner_recon}-real links) + FP32 arithmetic, delta {delta})")
    return {"workload": ("clover even-odd 16^3x32, kappa=0.1360, csw=1.0, links exp(i 0.3 H) "
                         f"(H GUE) 12-real, antiperiodic t; {how} to 1e-10 true residual"),
            "rhs_per_step": batch, "lattice": list(DIMS), "kappa": KAPPA, "csw": CSW,
            "l2": "flushed (256 MiB write) before every step"}


# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    from qphix_b200 import _lib
    from qphix_b200 import api

    B = args.batch
    inputs = make_inputs(DIMS, B, seed=2024 + 17 * rank)
    lat = api.Lattice(DIMS, device=local)
    stream = torch.cuda.Stream()
    lat.set_stream(stream.cuda_stream)
    # FP64 outer operator, inner operator on 16-bit storage
    u64 = lat.gauge("f64", 12).upload(inputs["gauge"])
    A64 = lat.clover("f64").upload(inputs["clov_odd"])
    Ai64 = lat.clover("f64").upload(inputs["invclov_even"])
    M64 = api.EvenOddCloverOperator(u64, A64, Ai64)
    ui = lat.gauge(args.inner, args.inner_recon).upload(inputs["gauge"])
    Ai = lat.clover(args.inner).upload(inputs["clov_odd"])
    Aii = lat.clover(args.inner).upload(inputs["invclov_even"])
    Mi = api.EvenOddCloverOperator(ui, Ai, Aii)
    d_rich = args.delta if args.solver == "richardson" else DEFAULT_DELTA["richardson"]
    d_ru = args.delta if args.solver == "ru" else DEFAULT_DELTA["ru"]
    rich = api.InvRichardsonMultiPrec(M64, Mi, "bicgstab", delta=d_rich, max_iters=100, inner_max_iters=5000)
    ru = api.InvBiCGStabMixed(M64, Mi, delta=d_ru, max_iters=20000)
    solver = ru if args.solver == "ru" else rich
    b_res = lat.spinor("f64", B).upload(inputs["rhs"])    # resident sources
    b = lat.spinor("f64", B)
    x = lat.spinor("f64", B)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step_resident():
        with torch.cuda.stream(stream):
            flush.fill_(1)
        api.copy(b, b_res)
        api.zero(x)
        return solver(x, b, RSD)

    # host buffers for the end-to-end path (pinned)
    h_rhs = torch.from_numpy(np.ascontiguousarray(
        np.stack([inputs["rhs"].real, inputs["rhs"].imag], axis=-1))).pin_memory()
    h_x = torch.empty_like(h_rhs).pin_memory()
    layout = api._canon_layout()
    import ctypes as C

    def step_e2e():
        with torch.cuda.stream(stream):
            flush.fill_(1)
        _lib.check(_lib._lib.qphix_gpu_field_upload(b.h, C.c_void_p(h_rhs.data_ptr()), C.byref(layout), -1, -1))
        api.zero(x)
        inf = solver(x, b, RSD)
        _lib.check(_lib._lib.qphix_gpu_field_download(x.h, C.c_void_p(h_x.data_ptr()), C.byref(layout), -1))
        return inf

    def barrier():
        if dist is not None:
            dist.barrier()

    def launches():
        n = C.c_ulonglong(0)
        _lib._lib.qphix_gpu_launch_count(C.byref(n))
        return n.value

    for _ in range(args.warmup):
        infos = step_resident()
    # ---- timed: resident inputs ------------------------------------------------
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = launches()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    all_infos = []
    for i in range(args.steps):
        ev[i][0].record(stream)
        all_infos.append(step_resident())
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    n_launch = launches() - l0
    clk = clocks.stop()
    step_ms = [a.elapsed_time(bb) for a, bb in ev]
    total_s = sum(step_ms) / 1e3
    if dist is not None:
        t = torch.tensor([total_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_s = float(t.item())
    value = world * B * args.steps / total_s
    worst_resid = max(i["true_rel_resid"] for inf in all_infos for i in inf)
    converged = all(i["status"] == 0 for inf in all_infos for i in inf)
    outer_iters = all_infos[-1][0]["n_iters"]
    mv_apps = all_infos[-1][0]["mv_apps"]

    # ---- e2e through the C ABI with host buffers -------------------------------
    step_e2e()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_ms = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        step_e2e()
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    e2e_total = sum(e2e_ms) / 1e3
    if dist is not None:
        t = torch.tensor([e2e_total], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * B * args.steps / e2e_total
    bytes_io = int(h_rhs.numel() * 8)

    # ---- the other mixed solver, for comparison --------------------------------
    other = rich if args.solver == "ru" else ru
    ots = []
    for _ in range(2):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        api.copy(b, b_res)
        api.zero(x)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        oinf = other(x, b, RSD)
        e1.record(stream)
        torch.cuda.synchronize()
        ots.append(e0.elapsed_time(e1))
    other_line = {"solver": "richardson" if args.solver == "ru" else "ru",
                  "delta": d_rich if args.solver == "ru" else d_ru,
                  "solves_per_s": round(B * 1e3 / min(ots), 3),
                  "worst_true_rel_resid": max(i["true_rel_resid"] for i in oinf),
                  "iters": oinf[0]["n_iters"], "mv_apps": oinf[0]["mv_apps"]}

    # ---- the same solver with a Q16 inner operator (16-bit fixed-point spinors
    # with per-site norms, FP16 links and clover) ---------------------------------
    q16_line = None
    if args.inner != "q16":
        uq = lat.gauge("q16", args.inner_recon).upload(inputs["gauge"])
        Aq = lat.clover("q16").upload(inputs["clov_odd"])
        Aiq = lat.clover("q16").upload(inputs["invclov_even"])
        Mq = api.EvenOddCloverOperator(uq, Aq, Aiq)
        sq = (api.InvRichardsonMultiPrec(M64, Mq, "bicgstab", delta=d_rich, max_iters=100, inner_max_iters=5000)
              if args.solver == "richardson" else api.InvBiCGStabMixed(M64, Mq, delta=d_ru, max_iters=20000))
        qts = []
        for _ in range(3):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            api.copy(b, b_res)
            api.zero(x)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            qinf = sq(x, b, RSD)
            e1.record(stream)
            torch.cuda.synchronize()
            qts.append(e0.elapsed_time(e1))
        q16_line = {"inner": "q16", "solver": args.solver, "solves_per_s": round(B * 1e3 / min(qts[1:]), 3),
                    "worst_true_rel_resid": max(i["true_rel_resid"] for i in qinf),
                    "iters": qinf[0]["n_iters"], "mv_apps": qinf[0]["mv_apps"]}

    # ---- plain FP64 BiCGStab beside it ------------------------------------------
    fp64 = fp64_1 = None
    if not args.no_fp64:
        bic = api.InvBiCGStab(M64, 5000)

        def time_fp64(bf, xf, reps):
            api.zero(xf)
            infs = bic(xf, bf, RSD)
            ts = []
            for _ in range(reps):
                with torch.cuda.stream(stream):
                    flush.fill_(1)
                api.zero(xf)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                infs = bic(xf, bf, RSD)
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            ms = statistics.median(ts)
            n = len(infs)
            return {"rhs_per_solve": n, "solves_per_s": n * 1e3 / ms, "ms_per_block": ms,
                    "iters": max(i["n_iters"] for i in infs),
                    "true_rel_resid": max(i["true_rel_resid"] for i in infs),
                    "status": max(i["status"] for i in infs)}
        # like for like: the same 8-rhs block the mixed solver takes
        fp64 = time_fp64(b_res, x, max(2, min(args.steps, 4)))
        b1 = lat.spinor("f64", 1).upload(inputs["rhs"][0])
        x1 = lat.spinor("f64", 1)
        fp64_1 = time_fp64(b1, x1, max(2, min(args.steps, 5)))

    # ---- roofline: the FP16 clover Dslash kernel (inner solve), L2 flushed ------
    def dslash_roofline(dims, prec, nrhs, n=20, achi=False, reduce=False):
        """One FP16 clover Dslash of the inner operator in the solve's launch
        configuration, timed alone with CUDA events on the lattice's stream,
        L2 flushed before every launch: A^-1 D psi (the operator's first
        kernel) or, with achi, A chi - b D psi on the odd checkerboard (its
        second kernel, the larger share of the solve); with reduce, carrying
        the reductions BiCGStab fuses into its t = M s launch (|t|^2 and
        <t, s>, folded on the device, no host round trip) as in the solve.
        Algorithmic bytes per site: nrhs x (input + output spinor, + chi) +
        8 links (12 reals) + the packed clover term (72 reals)."""
        from qphix_b200 import fields as F
        lat2 = lat if dims == DIMS else api.Lattice(dims, device=local)
        if dims != DIMS:
            lat2.set_stream(stream.cuda_stream)
        # a larger lattice: the C2 links tiled (link values do not change timing)
        g = inputs["gauge"] if dims == DIMS else np.tile(inputs["gauge"], (1, 1, F.vh(dims) // F.vh(DIMS), 1, 1))
        u = lat2.gauge(prec, 12).upload(g)
        ckey = "clov_odd" if achi else "invclov_even"
        cl = lat2.clover(prec).upload(inputs[ckey] if dims == DIMS else
                                      np.tile(inputs[ckey][:1], (F.vh(dims), 1, 1)))
        psi = lat2.spinor(prec, nrhs).upload(np.stack([F.gaussian_spinor(dims, 3 + i) for i in range(nrhs)]))
        out = lat2.spinor(prec, nrhs)
        chi = (lat2.spinor(prec, nrhs).upload(np.stack([F.gaussian_spinor(dims, 40 + i) for i in range(nrhs)]))
               if achi else None)
        D = api.ClovDslash(lat2, -1.0, 1.0, 1.0)

        def launch():
            if achi and reduce:
                D.dslashAChiMinusBDPsiNorms(out, psi, chi, u, cl, 0.25, 1, 1, fetch=False)
            elif achi:
                D.dslashAChiMinusBDPsi(out, psi, chi, u, cl, 0.25, 1, 1)
            else:
                D.dslash(out, psi, u, cl, 1, 0)
        for _ in range(3):
            launch()
        durs = []
        for _ in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            launch()
            e1.record(stream)
            torch.cuda.synchronize()
            durs.append(e0.elapsed_time(e1) / 1e3)
        vh = F.vh(dims)
        esize = {"f16": 2, "bf16": 2, "q16": 2, "q16f32": 2, "f32": 4, "f64": 8}[prec]
        lsize = 4 if prec == "q16f32" else esize  # links and clover
        norm = 4 if prec in ("f16", "bf16", "q16", "q16f32") else 0
        per_site = nrhs * (3 if achi else 2) * (24 * esize + norm) + 8 * 12 * lsize + 72 * lsize
        t = statistics.mean(durs)
        return per_site, vh, t

    peak, peak_kind = peaks()
    per_site, vh, t = dslash_roofline(DIMS, args.inner, B, achi=True, reduce=True)
    _, _, t_nored = dslash_roofline(DIMS, args.inner, B, achi=True)
    achieved = per_site * vh / t / 1e9
    traffic = profile_traffic().get(f"clover_achi_{args.inner}_12_{'x'.join(map(str, DIMS))}_n{B}")
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": (round(traffic * vh) if traffic else None),
            "kernel": f"clover Dslash A chi - b D psi, {args.inner} storage, 12-real links, {B} rhs per launch "
                      f"(the inner operator's second kernel and the solve's largest share), with the |t|^2 and "
                      f"<t, s> reductions fused into it as in the solve; traffic from the in-solve launch",
            "bytes_per_site": per_site, "sites": vh, "nrhs": B, "launch_us": round(t * 1e6, 2),
            "launch_us_without_reductions": round(t_nored * 1e6, 2),
            "note": "the 16^3x32 working set fits in L2 within a solve; L2 is flushed before each timed launch"}
    ps1, _, t1 = dslash_roofline(DIMS, args.inner, B)
    traffic1 = profile_traffic().get(f"clover_dslash_{args.inner}_12_{'x'.join(map(str, DIMS))}_n{B}")
    roof_first = {"kernel": f"clover Dslash A^-1 D psi, {args.inner} storage, {B} rhs (the operator's first kernel)",
                  "bytes_per_site": ps1, "achieved": round(ps1 * vh / t1 / 1e9, 1),
                  "frac": round(ps1 * vh / t1 / 1e9 / peak, 4), "launch_us": round(t1 * 1e6, 2),
                  "traffic": (round(traffic1 * vh) if traffic1 else None)}
    big = (32, 32, 32, 64)
    ps2, vh2, t2 = dslash_roofline(big, args.inner, 1, n=10)
    traffic2 = profile_traffic().get(f"clover_dslash_{args.inner}_12_32x32x32x64_n1")
    roof_big = {"lattice": list(big), "nrhs": 1, "bytes_per_site": ps2, "achieved": round(ps2 * vh2 / t2 / 1e9, 1),
                "frac": round(ps2 * vh2 / t2 / 1e9 / peak, 4), "launch_us": round(t2 * 1e6, 1),
                "traffic": (round(traffic2 * vh2) if traffic2 else None)}
    # the same A^-1 D psi launch with FP32 and FP64 storage (the FP64 outer
    # operator's and the FP32 configurations' kernel), HBM-bound at this size
    for wide in ("f32", "f64"):
        psw, vhw, tw = dslash_roofline(big, wide, 1, n=10)
        roof_big[wide] = {"bytes_per_site": psw, "achieved": round(psw * vhw / tw / 1e9, 1),
                          "frac": round(psw * vhw / tw / 1e9 / peak, 4), "launch_us": round(tw * 1e6, 1)}

    cpu = None
    extra = None
    if rank == 0 and world == 1:
        try:
            cpu = cpu_baseline_leg(inputs, DIMS)
        except Exception as e:  # pragma: no cover
            cpu = {"value": None, "error": str(e)}
        if not args.no_extra:
            extra = extra_configs()

    if rank == 0:
        p = sorted(step_ms)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_s * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": f"mixed: f64 outer, f32 arithmetic on {args.inner} storage inner",
            "data": "synthetic (seeded)", "config": config_dict(B, args.inner, args.solver, args.inner_recon, args.delta),
            "e2e": {"value": round(e2e_value, 3), "unit": "solves/s", "h2d_bytes_per_step": bytes_io,
                    "d2h_bytes_per_step": bytes_io},
            "roofline": roof, "roofline_first_kernel": roof_first, "roofline_large_lattice": roof_big,
            "cpu_baseline": cpu, "gpu_launches": int(n_launch),
            "clocks": clk,
            "p50_ms_per_step": round(p[len(p) // 2], 3), "p99_ms_per_step": round(p[min(len(p) - 1, int(0.99 * len(p)))], 3),
            "fp64_plain": fp64,
            "mixed_vs_fp64_solves_ratio": (round(value / world / fp64["solves_per_s"], 3) if fp64 else None),
            "fp64_plain_1rhs": fp64_1,
            "mixed_vs_fp64_1rhs_solves_ratio": (round(value / world / fp64_1["solves_per_s"], 3) if fp64_1 else None),
            "solver": {"kind": "bicgstab_reliable_update" if args.solver == "ru" else "richardson_bicgstab",
                       "delta": args.delta, "iters": outer_iters, "mv_apps": mv_apps,
                       "worst_true_rel_resid": worst_resid, "all_converged": converged},
            "other_mixed_solver": other_line,
            "q16_inner": q16_line,
            "q16_inner_vs_fp64_solves_ratio": (round(q16_line["solves_per_s"] / fp64["solves_per_s"], 3)
                                               if (fp64 and q16_line) else None),
        }
        if extra:
            sv = extra.get("serve", {})
            line["serve_latency_p50_ms"] = sv.get("latency_p50_ms")
            line["serve_latency_p99_ms"] = sv.get("latency_p99_ms")
            line["serve_solves_per_s"] = sv.get("solves_per_s")
            line["configs"] = extra
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
