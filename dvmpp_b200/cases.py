"""Command-line drivers for the standalone workloads.

    python -m dvmpp_b200.cases nbody --n 1048576 [--prec f32|f64|both] [--reps 3]

nbody: the standalone regularised Biot-Savart workload -- N blobs, 70 % in a
wake x ~ U[0.5, 20], z ~ N(0, 1), 30 % in the annulus 0.5 < r < 1.5,
Gamma ~ N(0, 1e-3) summing to zero, sigma = 0.081880 (ds^0.675 of the
128-panel R = 0.5 circle), seed 2.  Prints one JSON line with the pair
kernel's CUDA-event time, pairs/s, FP32-pipe fraction and (with both
precisions) the FP32-vs-FP64 error.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import native as N
from . import workloads as W

SIGMA_CYL128 = 0.08188040878164335


def _fp32_peak_tflops(sms: int) -> float:
    mhz = 1965.0
    try:
        here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        with open(os.path.join(here, "MEASURED_PEAKS.json")) as f:
            mhz = float(json.load(f).get("sm_max_mhz", mhz))
    except (OSError, ValueError):
        pass
    return sms * 128 * 2 * mhz * 1e6 / 1e12


def run_nbody(n: int, precs, reps: int, seed: int = 2):
    ctx = N.Context(0)
    sms, _, _ = ctx.device_info()
    x, z, g, s = W.wake(n, seed, SIGMA_CYL128)
    bx, bz = W.circle(128)
    out = {"workload": "nbody", "n": n, "pairs": n * (n - 1), "results": {}}
    fields = {}
    for prec in precs:
        p = N.Params(capacity=n, precision=prec, rng=N.RNG_PHILOX)
        sim = ctx.sim(p, bx, bz)
        sim.set_blobs(x, z, g, s)
        sim.phase(N.PHASE_BIOTSAVART)  # warm-up
        ctx.set_profiling(True)
        ctx.profile_reset()
        for _ in range(reps):
            sim.phase(N.PHASE_BIOTSAVART)
        prof = ctx.profile()
        ctx.set_profiling(False)
        ms = prof["nbody"][0] / max(prof["nbody"][1], 1)
        d = sim.blobs()
        fields[prec] = (d["u"], d["w"])
        tf = 12.0 * n * (n - 1) / (ms / 1e3) / 1e12
        out["results"]["f32" if prec == N.F32 else "f64"] = {
            "pair_kernel_ms": ms, "sort_pack_combine_ms": prof["sort"][0] / max(prof["sort"][1], 1),
            "gpairs_per_s": n * (n - 1) / (ms / 1e3) / 1e9, "tflops_12_per_pair": tf,
            "fp32_peak_frac": tf / _fp32_peak_tflops(sms)}
        sim.close()
    if N.F32 in fields and N.F64 in fields:
        (uf, wf), (ud, wd) = fields[N.F32], fields[N.F64]
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        out["f32_vs_f64"] = {"rel_l2_u": rel(uf, ud), "rel_l2_w": rel(wf, wd),
                             "max_rel_u": float(np.max(np.abs(uf - ud)) / np.max(np.abs(ud))),
                             "max_rel_w": float(np.max(np.abs(wf - wd)) / np.max(np.abs(wd)))}
    ctx.close()
    return out


def serve_params(r) -> N.Params:
    """Parameters of one serving request (Philox walk, FP32 pair sums, REFLECT);
    capacity: the blobs its steps can release, with a 2x margin."""
    M = 3
    return N.Params(nu=r["nu"], ux=r["ux"], dt=0.005, max_numpanelvort=M, rng=N.RNG_PHILOX,
                    precision=N.F32, seed=r["seed"], surface_cross=N.REFLECT,
                    capacity=r["steps"] * (M + 1) * r["npanels"] * 2 + 1024)


def run_serving(count: int, seed: int, rate: float, steps_range, panels_range, max_active: int,
                budget_gb: float, realtime: bool, serial_too: bool, graph: bool = True,
                sync: bool = True):
    """The serving workload, continuous batching and (optionally) the plain
    serial path on the same requests; returns both summaries."""
    reqs = W.serving_requests(count, seed, rate, steps_range, panels_range)
    out = {"workload": "serving", "requests": count, "rate_per_s": rate,
           "steps_range": list(steps_range), "panels_range": list(panels_range),
           "budget_gb": budget_gb, "realtime": realtime}
    modes = [("batched", False)] + ([("serial", True)] if serial_too else [])
    for name, serial in modes:
        ctx = N.Context(0)
        srv = N.Server(ctx, budget_bytes=int(budget_gb * 2**30), max_active=max_active)
        srv.set_option(N.SERVE_GRAPH, 1 if graph else 0)
        srv.set_option(N.SERVE_SYNC, 1 if sync else 0)
        for r in reqs:
            srv.submit(serve_params(r), *r["body"], r["steps"], r["arrival"])
        srv.run(serial=serial, realtime=realtime)
        out[name] = srv.stats()
        srv.close()
        ctx.close()
    if serial_too:
        out["speedup_sim_steps"] = (out["batched"]["sim_steps_per_s"]
                                    / max(out["serial"]["sim_steps_per_s"], 1e-12))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    nb = sub.add_parser("nbody")
    nb.add_argument("--n", type=int, default=1 << 20)
    nb.add_argument("--prec", choices=["f32", "f64", "both"], default="f32")
    nb.add_argument("--reps", type=int, default=3)
    nb.add_argument("--seed", type=int, default=2)
    sv = sub.add_parser("serve")
    sv.add_argument("--requests", type=int, default=100)
    sv.add_argument("--seed", type=int, default=7)
    sv.add_argument("--rate", type=float, default=20.0)
    sv.add_argument("--steps", type=int, nargs=2, default=[100, 2000])
    sv.add_argument("--panels", type=int, nargs=2, default=[64, 512])
    sv.add_argument("--max-active", type=int, default=256)
    sv.add_argument("--budget-gb", type=float, default=150.0)
    sv.add_argument("--realtime", action="store_true")
    sv.add_argument("--serial", action="store_true", help="also run the plain serial path")
    sv.add_argument("--no-graph", action="store_true")
    sv.add_argument("--no-sync", action="store_true")
    a = ap.parse_args(argv)
    if a.cmd == "serve":
        print(json.dumps(run_serving(a.requests, a.seed, a.rate, tuple(a.steps), tuple(a.panels),
                                     a.max_active, a.budget_gb, a.realtime, a.serial,
                                     not a.no_graph, not a.no_sync)))
    if a.cmd == "nbody":
        precs = {"f32": [N.F32], "f64": [N.F64], "both": [N.F32, N.F64]}[a.prec]
        print(json.dumps(run_nbody(a.n, precs, a.reps, a.seed)))


if __name__ == "__main__":
    main()
