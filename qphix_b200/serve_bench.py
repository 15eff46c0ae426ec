"""Serving benchmark: a seeded stream of solve requests through the server.

    python -m qphix_b200.serve_bench [--requests 2000] [--load 0.7] [--slots 4]

Workload (seeded): lattice volume uniform over 8^4, 16^3x32, 24^3x48,
32^3x64; operator uniform over Wilson, clover (c_sw = 1.0) and twisted mass
(mu = 0.01); kappa uniform in [0.120, 0.136]; a pool of 4 gauge fields per
volume (links exp(i 0.3 H), H seeded GUE, 12-real on the device), resident in
the server; 1-12 Gaussian right-hand sides per request (drawn from a pool of
12 seeded sources per volume); every request solved to a 1e-10 FP64 true
residual with FP16-storage iterations and FP64 reliable updates.

Capacity is measured first, closed loop (a burst of requests submitted at
once, completions per second of wall time); the open-loop run then submits
`--requests` requests at Poisson arrival times with mean rate `--load` x
capacity and reports the latency (submit to solution in the caller's
buffer, from the server's own clock) p50 / p99, and solves/s (right-hand
sides solved per second of wall time).  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import sys
import threading
import time

import numpy as np

VOLUMES = [(8, 8, 8, 8), (16, 16, 16, 32), (24, 24, 24, 48), (32, 32, 32, 64)]
OPS = ["wilson", "clover", "tm"]
MU = 0.01
CSW = 1.0


def make_requests(n, seed, nvol=len(VOLUMES)):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        out.append(dict(vol=int(rng.integers(nvol)), ens=int(rng.integers(4)), op=OPS[int(rng.integers(3))],
                        kappa=float(rng.uniform(0.120, 0.136)), nrhs=int(rng.integers(1, 13)),
                        src=int(rng.integers(12))))
    return out


def main(argv=None):
    print(json.dumps(run(argv)), flush=True)


def run(argv=None):
    """Runs the benchmark (arguments as on the command line) and returns its
    result line as a dict."""
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=300)
    ap.add_argument("--load", type=float, default=0.7)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--calibrate", type=int, default=48)
    ap.add_argument("--seed", type=int, default=2025)
    ap.add_argument("--volumes", type=int, default=4, help="use the first N volumes of the list (quick runs)")
    ap.add_argument("--solver", default="ru", choices=["ru", "richardson"],
                    help="ru: BiCGStab with reliable updates (delta 0.1); richardson: InvRichardsonMultiPrec "
                         "(delta 0.005)")
    args = ap.parse_args(argv)
    vols = VOLUMES[:args.volumes]

    from . import api
    from . import fields as F

    t0 = time.perf_counter()
    srv = api.Server(int(args.budget_gb * (1 << 30)), slots=args.slots, low_prec="f16", solver=args.solver,
                     delta=0.005 if args.solver == "richardson" else 0.1)
    ens = {}
    sources = {}
    for v, dims in enumerate(vols):
        for e in range(4):
            g = F.make_gauge(dims, 7000 + 10 * v + e, "exp", eps=0.3)
            ens[(v, e)] = srv.add_ensemble(dims, g)
            del g
        # 12 sources, stored twice over so that any run of <= 12 consecutive
        # ones is a contiguous slice of the interleaved C layout
        pool = api.Server.interleave(np.stack([F.gaussian_spinor(dims, 9000 + 100 * v + k) for k in range(12)]))
        sources[v] = np.concatenate([pool, pool])
    setup_s = time.perf_counter() - t0

    # solution buffers, recycled once a request has been collected
    free = {}
    lock = threading.Lock()

    def take(v, n):
        with lock:
            lst = free.get((v, n))
            if lst:
                return lst.pop()
        return np.empty((n,) + sources[v].shape[1:])

    def give(v, buf):
        with lock:
            free.setdefault((v, buf.shape[0]), []).append(buf)

    def submit(q):
        x = take(q["vol"], q["nrhs"])
        t = srv.submit(ens[(q["vol"], q["ens"])], q["op"], sources[q["vol"]][q["src"]:q["src"] + q["nrhs"]],
                       F.kappa_to_mass(q["kappa"]), CSW, MU, rsd_target=1e-10, max_iters=20000, out=x)
        return t, q["vol"]

    def collect(tickets, n, results):
        # waits in submission order, as tickets arrive; frees each buffer
        for i in range(n):
            while len(tickets) <= i:
                time.sleep(0.0005)
            t, v = tickets[i]
            x, info = srv.wait(t, raise_on_error=False, as_complex=False)
            give(v, x)
            results.append(info)
            if (i + 1) % 100 == 0:
                print(f"[serve] {i + 1}/{n} collected", file=sys.stderr, flush=True)

    # closed-loop capacity (also warms the shape autotuner and graph paths)
    cal = make_requests(args.calibrate, args.seed + 1, len(vols))
    t0 = time.perf_counter()
    cal_t = [submit(q) for q in cal]
    cal_res = []
    collect(cal_t, len(cal_t), cal_res)
    cap_s = time.perf_counter() - t0
    capacity = args.calibrate / cap_s
    print(f"[serve] setup {setup_s:.0f} s, capacity {capacity:.2f} requests/s", file=sys.stderr, flush=True)
    cap_rhs = sum(q["nrhs"] for q in cal) / cap_s

    # open loop: Poisson arrivals at load x capacity
    reqs = make_requests(args.requests, args.seed, len(vols))
    rng = np.random.default_rng(args.seed + 2)
    rate = args.load * capacity
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
    tickets, results = [], []
    collector = threading.Thread(target=collect, args=(tickets, len(reqs), results))
    start = time.perf_counter()
    collector.start()
    for q, at in zip(reqs, arrivals):
        now = time.perf_counter() - start
        if at > now:
            time.sleep(at - now)
        tickets.append(submit(q))
    collector.join()
    wall = time.perf_counter() - start
    st = srv.stats()
    srv.close()

    lat = np.array([r["latency_s"] for r in results])
    solve = np.array([r["solve_s"] for r in results])
    queue = np.array([r["queue_s"] for r in results])
    ok = [r["status"] == 0 for r in results]
    nrhs = sum(q["nrhs"] for q in reqs)
    by_vol = {}
    for q, r in zip(reqs, results):
        k = "x".join(map(str, VOLUMES[q["vol"]]))
        by_vol.setdefault(k, []).append(r["latency_s"])
    line = {
        "metric": "serving: solve latency p50 / p99 and solves/s under Poisson arrivals",
        "volumes": ["x".join(map(str, d)) for d in vols], "requests": len(reqs), "rhs_solved": nrhs, "load": args.load, "slots": args.slots,
        "capacity_requests_per_s": capacity, "capacity_rhs_per_s": cap_rhs,
        "arrival_rate_per_s": rate, "wall_s": wall,
        "solves_per_s": nrhs / wall, "requests_per_s": len(reqs) / wall,
        "latency_p50_ms": float(np.percentile(lat, 50) * 1e3), "latency_p99_ms": float(np.percentile(lat, 99) * 1e3),
        "solve_p50_ms": float(np.percentile(solve, 50) * 1e3), "queue_p99_ms": float(np.percentile(queue, 99) * 1e3),
        "latency_p50_ms_by_volume": {k: float(np.percentile(v, 50) * 1e3) for k, v in by_vol.items()},
        "latency_p99_ms_by_volume": {k: float(np.percentile(v, 99) * 1e3) for k, v in by_vol.items()},
        "all_converged": all(ok), "failed": len(ok) - sum(ok),
        "worst_true_rel_resid": max(r["true_rel_resid"] for r in results),
        "server": st, "setup_s": setup_s,
        "data": "synthetic (seeded)",
        "solver": args.solver,
    }
    return line


if __name__ == "__main__":
    main()
