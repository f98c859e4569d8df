#!/usr/bin/env python
"""Benchmark of the batched DVM step on B200.

Workload ("batched", the metric's configuration): 64 independent bodies --
circle R=0.5, ellipses of aspect U[1,4], rounded squares (side 1, corner
radius 0.05) -- with panel counts log-uniform in [64, 512], each pre-seeded
with a wake of log-uniform 1e4..4e5 blobs (seeded synthetic data), Euler,
dt = 0.005, nu = 1e-3, ux = 1, REFLECT, FP32 compensated pair sums.

A "step" advances all 64 simulations by one time step (DVMBase::compute_step
each); value = simulation-steps per second over the whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  Multi-GPU runs are replicas (each rank runs its own
copy of the batch; no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched sim-steps/s vs plain GPU at <=1e-5 rel vel err; p50/p99 latency"
UNIT = "sim-steps/s"


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ---------------------------------------------------------------------------
# distributed plumbing (replicas: only timing values cross ranks)
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = _env_int("WORLD_SIZE", 1)
        self.rank = _env_int("RANK", 0)
        self.local = _env_int("LOCAL_RANK", 0)
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="dvm_clocks_", suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [q.strip() for q in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def make_instances(count: int, seed: int):
    from dvmpp_b200 import workloads as W

    return W.batched_instances(count, seed)


def sim_params(inst, steps_total: int, prepush_steps: int, async_steps: int = 0):
    """async_steps: room for that many per-step pushes on top of the prepushed
    uniforms (asynchronous pushes append without compacting the stream)."""
    from dvmpp_b200 import native as N

    M = 3
    grow = steps_total * (M + 1) * inst["npanels"] * 2  # release counts can exceed (M+1)
    cap = inst["nblobs"] + grow
    per_step = 2 * cap + 2 * (M + 1) * inst["npanels"]
    push_ub = 2 * (cap + 2 * (M + 1) * inst["npanels"]) + 2 * (M + 1) * inst["npanels"] + 64
    return N.Params(rho=1.0, nu=1e-3, dt=0.005, ux=1.0, uz=0.0, cutoff_exp=0.675,
                    max_numpanelvort=M, scheme=N.EULER, surface_cross=N.REFLECT,
                    rng=N.RNG_INJECT, precision=N.F32, seed=1, capacity=cap,
                    rng_capacity=prepush_steps * per_step + 1024 + async_steps * push_ub)


def pinned(n: int):
    """A pinned host float64 buffer (torch allocates it; numpy views it)."""
    import torch

    return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()


def uniforms_for(sims, rng, steps: int):
    """(0,1] uniforms covering `steps` steps of every simulation."""
    out = []
    for s in sims:
        n = s.n_hint
        need = steps * (2 * n + 2 * (3 + 1) * s.np + 64)
        out.append(1.0 - rng.random(need))
    return out


# ---------------------------------------------------------------------------
# the reference arm / CPU baseline: the reference's own code, phase-timed on
# a sample of the instances and extrapolated by each phase's complexity
# ---------------------------------------------------------------------------
def _cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class RefModel:
    """Per-phase cost rates of the reference step, measured on sampled
    instances and interpolated (linearly in log N, clamped at the ends) to
    every instance of the batch: biotsavart ~ N^2, vortexsheetbc ~ N Np
    (serial in the reference), solvevortexsheet ~ N Np, diffusion + crossing
    ~ N, release + loads ~ Np."""

    KEYS = ("a", "b", "c", "d", "e")

    def __init__(self):
        self.samples = []  # (N, Np, rates)

    def add(self, N, Np, t):
        N, Np = max(N, 1), max(Np, 1)
        self.samples.append((N, Np, {"a": t["bs"] / (N * N), "b": t["sbc"] / (N * Np),
                                     "c": t["solve"] / (N * Np), "d": (t["diff"] + t["cross"]) / N,
                                     "e": (t["rel"] + t["loads"]) / Np}))
        self.samples.sort(key=lambda r: r[0])

    def rates_at(self, N) -> dict:
        xs = [math.log(r[0]) for r in self.samples]
        lx = math.log(max(N, 1))
        return {k: float(np.interp(lx, xs, [r[2][k] for r in self.samples])) for k in self.KEYS}

    def phase_times(self, instances) -> dict:
        """Seconds per batched step by phase of DVMBase::compute_step."""
        out = {"biotsavart_N2": 0.0, "vortexsheetbc_NNp": 0.0, "solve_NNp": 0.0,
               "diffusion_and_crossing_N": 0.0, "release_and_loads_Np": 0.0}
        for inst in instances:
            N, Np = inst["nblobs"], inst["npanels"]
            r = self.rates_at(N)
            out["biotsavart_N2"] += r["a"] * N * N
            out["vortexsheetbc_NNp"] += r["b"] * N * Np
            out["solve_NNp"] += r["c"] * N * Np
            out["diffusion_and_crossing_N"] += r["d"] * N
            out["release_and_loads_Np"] += r["e"] * Np
        return out

    def step_time(self, instances) -> float:
        return sum(self.phase_times(instances).values())

    def table(self):
        return [{"N": n, "Np": m, "s_per_pair_biotsavart": r["a"], "s_per_pair_sheetbc": r["b"],
                 "s_per_pair_solve": r["c"], "s_per_blob_diff_cross": r["d"],
                 "s_per_panel_release_loads": r["e"]} for n, m, r in self.samples]


REF_SUBSET = 4096       # targets / blobs of the sub-sampled phases on large instances
REF_FULL_MAX = 200_000  # instances up to this size run the whole reference step


def _ref_params():
    from oracle.pyoracle import SimParams

    return SimParams(rho=1.0, nu=1e-3, dt=0.005, ux=1.0, uz=0.0, cutoff_exp=0.675,
                     max_numpanelvort=3, scheme="euler", surface_cross="REFLECT", seed=1, steps=10)


def _timed_phases(s, keys_phases):
    t = {}
    for key, phase in keys_phases:
        t0 = time.perf_counter()
        s.phase(phase)
        t[key] = time.perf_counter() - t0
    return t


def ref_sample_step(ref, inst, workdir):
    """The reference's DVMBase::compute_step phases on one instance, timed with
    the host clock (output writing is not part of it), as seconds for the
    whole instance.  Up to REF_FULL_MAX blobs every phase runs on the whole
    instance.  Larger instances are sampled (the N-proportional phases on a
    subset): biotsavart as the reference's own computeInducedAt at REF_SUBSET
    randomly chosen blobs against all N sources (the same pair loop as
    computeSelfInduced) scaled by N / REF_SUBSET; vortexsheetbc, diffusion and
    crossing on a REF_SUBSET-blob subset scaled likewise; solvevortexsheet as
    its blob-free part (the normal-equations solve) plus the subset's
    right-hand-side part scaled; release and loads as measured."""
    p = _ref_params()
    bx, bz = inst["body"]
    x, z, g, sg = inst["blobs"]
    N = x.size
    order = [("bs", 0), ("solve", 1), ("sbc", 2), ("diff", 4), ("rel", 5), ("cross", 6),
             ("loads", 7)]
    if N <= REF_FULL_MAX:
        s = ref.sim(p, bx, bz, workdir=workdir)
        s.set_blobs(x, z, g, sg)
        t = _timed_phases(s, order)
        del s
        t["how"] = "full"
        return t
    rng = np.random.default_rng(N)
    pick = np.sort(rng.choice(N, REF_SUBSET, replace=False))
    t0 = time.perf_counter()
    ref.direct_at(x, z, g, sg, x[pick], z[pick])
    scale = N / REF_SUBSET
    t = {"bs": (time.perf_counter() - t0) * scale}
    s0 = ref.sim(p, bx, bz, workdir=workdir)  # no blobs: the solve's N-free part
    t_solve0 = _timed_phases(s0, [("solve", 1)])["solve"]
    del s0
    s = ref.sim(p, bx, bz, workdir=workdir)
    s.set_blobs(x[pick], z[pick], g[pick], sg[pick])
    ts = _timed_phases(s, order[1:])
    del s
    t["solve"] = t_solve0 + max(ts["solve"] - t_solve0, 0.0) * scale
    for k in ("sbc", "diff", "cross"):
        t[k] = ts[k] * scale
    t["rel"], t["loads"] = ts["rel"], ts["loads"]
    t["how"] = f"subset {REF_SUBSET}"
    return t


def reference_sample(instances, quantiles):
    """One reference compute_step on the instances at the given size quantiles
    (0 = smallest, 1 = largest) and the per-phase rates interpolated to the
    whole batch."""
    from oracle.pyoracle import Ref, have_ref

    if not have_ref():
        return None
    ref = Ref()
    order = sorted(range(len(instances)), key=lambda k: instances[k]["nblobs"])
    pick = sorted({order[round(q * (len(order) - 1))] for q in quantiles},
                  key=lambda k: instances[k]["nblobs"])
    model = RefModel()
    total = 0.0
    how = []
    with tempfile.TemporaryDirectory(prefix="dvmref_") as wd:
        for k in pick:
            inst = instances[k]
            t0 = time.perf_counter()
            tt = ref_sample_step(ref, inst, wd)
            total += time.perf_counter() - t0
            model.add(inst["nblobs"], inst["npanels"], tt)
            how.append({"N": inst["nblobs"], "Np": inst["npanels"], "how": tt["how"]})
    batch = model.step_time(instances)
    return {"batch_step_s": batch, "sampled": how, "wall_s": total,
            "phases_s": model.phase_times(instances), "rates": model.table()}


REF_SAMPLE_NOTE = ("DVMBase::compute_step phases of the reference, timed per phase (output "
                   "writing off; the O(N) position update of convect not timed); instances up "
                   f"to {REF_FULL_MAX} blobs run whole, larger ones on {REF_SUBSET}-blob "
                   "subsets (biotsavart as computeInducedAt at that many targets against all "
                   "sources) scaled by N / subset; per-phase rates interpolated in log N "
                   "across the sampled sizes to all instances")


def run_reference_arm(args, dist):
    if dist.rank != 0:
        return
    instances = make_instances(args.instances, args.seed)
    from oracle.pyoracle import have_ref

    kind = "reference" if have_ref() else "port"
    if kind != "reference":
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libdvmref.so (the reference built from source) is absent"}))
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(_cores()))
    for _ in range(args.warmup):
        reference_sample(instances, [0.0])
    times = []
    phases = []
    r = None
    for k in range(args.steps):
        r = reference_sample(instances, [0.0, 0.5, 1.0])
        times.append(r["batch_step_s"])
        phases.append(r["phases_s"])
    step_s = float(np.median(times))
    value = args.instances / step_s
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": "batched: 64 mixed bodies (circle / ellipse aspect U[1,4] / "
                               "rounded square), panels log-U[64,512], wakes log-U[1e4,4e5] "
                               "blobs, Euler dt=0.005, REFLECT", "instances": args.instances,
                   "parallelism": "OpenMP host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": _cores(), "kind": kind,
                         "sample": "each step: the smallest, the median and the largest "
                                   "instance; " + REF_SAMPLE_NOTE,
                         "sampled": r["sampled"] if r else [],
                         "rates_last_step": r["rates"] if r else [],
                         "s_per_step_by_phase": {k: float(np.median([p[k] for p in phases]))
                                                 for k in phases[0]} if phases else {}},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def committed_traffic():
    """DRAM bytes per pair-kernel launch on this workload, from the committed
    ncu summary (one capture of the first timed step)."""
    try:
        with open(os.path.join(ROOT, "profiles", "bench_batched64_launches.md")) as f:
            for ln in f:
                if ln.strip().startswith("dram_bytes_per_launch:"):
                    return float(ln.split(":")[1])
    except (OSError, ValueError):
        pass
    return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


ACC_REL_L2 = 1e-5     # the metric's velocity bound, per field and per simulation
ACC_FORCE_REL = 5e-3  # Cd / Cl within 0.5 % (of the force coefficient's magnitude)


def _rel(a, b):
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a - b))


def _max_rel(a, b):
    mb = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / mb if mb > 0 else 0.0


def evaluate(sim, N):
    """Velocity fields, panel strengths and loads of a simulation's current
    state, without moving it: biotsavart, solvevortexsheet, vortexsheetbc
    (no convection) and compute_loads through the phase API."""
    for ph in (N.PHASE_BIOTSAVART, N.PHASE_SOLVE, N.PHASE_SHEETBC, N.PHASE_LOADS):
        sim.phase(ph)
    d = sim.blobs()
    return d, sim.gamma(), sim.loads()


def accuracy_vs_f64(ctx, sims, bodies, params):
    """The timed FP32-compensated arithmetic against FP64 on the identical
    state of every simulation of the batch: each FP32 simulation evaluates its
    current state in place (the same kernels and source chunking as its
    batched step); an FP64 copy of that state (same body and capacity) does
    the same in the reference's operation order.  Per simulation: rel-L2 and
    max-norm errors of u, w (blob-on-blob), uvs, wvs (sheet-on-blob), the total
    induced velocity (u + uvs, w + wvs) and gamma; Cd and Cl errors relative to
    the force coefficient's magnitude |(Cd, Cl)|."""
    from dvmpp_b200 import native as N

    fields = ("u", "w", "uvs", "wvs")
    per = []
    sq = {k: [0.0, 0.0] for k in fields + ("vel_total", "gamma")}
    for sim, (bx, bz), p in zip(sims, bodies, params):
        d32, g32, l32 = evaluate(sim, N)
        p64 = N.Params(**{**p.__dict__, "precision": N.F64, "rng": N.RNG_PHILOX})
        ref = ctx.sim(p64, bx, bz)
        ref.set_blobs(d32["x"], d32["z"], d32["circ"], d32["sigma"])
        d64, g64, l64 = evaluate(ref, N)
        ref.close()
        row = {"n": int(d32["x"].size), "np": int(g32.size)}
        pairs = [(k, d32[k], d64[k]) for k in fields]
        pairs.append(("vel_total", np.concatenate([d32["u"] + d32["uvs"], d32["w"] + d32["wvs"]]),
                      np.concatenate([d64["u"] + d64["uvs"], d64["w"] + d64["wvs"]])))
        pairs.append(("gamma", g32, g64))
        for k, a, b in pairs:
            row[k + "_rel_l2"] = _rel(a, b)
            row[k + "_max"] = _max_rel(a, b)
            sq[k][0] += float(np.sum((a - b) ** 2))
            sq[k][1] += float(np.sum(b ** 2))
        cmag = math.hypot(l64[2], l64[3])
        row["cd_f32"], row["cd_f64"], row["cl_f32"], row["cl_f64"] = l32[2], l64[2], l32[3], l64[3]
        row["cd_err"] = abs(l32[2] - l64[2]) / cmag if cmag > 0 else 0.0
        row["cl_err"] = abs(l32[3] - l64[3]) / cmag if cmag > 0 else 0.0
        per.append(row)
    worst = {k + "_rel_l2": max(r[k + "_rel_l2"] for r in per) for k in sq}
    worst.update({k + "_max": max(r[k + "_max"] for r in per) for k in sq})
    worst["cd_err"] = max(r["cd_err"] for r in per)
    worst["cl_err"] = max(r["cl_err"] for r in per)
    pooled = {k: math.sqrt(v[0] / v[1]) if v[1] > 0 else 0.0 for k, v in sq.items()}
    ok = (all(worst[k + "_rel_l2"] <= ACC_REL_L2 for k in sq)
          and worst["cd_err"] <= ACC_FORCE_REL and worst["cl_err"] <= ACC_FORCE_REL)
    return {"simulations": len(per), "blobs": int(sum(r["n"] for r in per)),
            "how": "FP32 step arithmetic vs FP64 (reference operation order) on the identical "
                   "state of every simulation after the timed steps; rel-L2 per simulation (worst "
                   "shown) and pooled over all blobs; Cd / Cl error relative to |(Cd, Cl)| of FP64",
            "bounds": {"rel_l2": ACC_REL_L2, "cd_cl": ACC_FORCE_REL},
            "worst": worst, "pooled_rel_l2": pooled, "within_bounds": bool(ok),
            "per_simulation": per}


def run_f64(ctx, instances, steps_total, warmup, steps):
    """The same batch with every pair sum in FP64 (reference operation order):
    fresh simulations from the same initial state, Philox walk; graph-replayed
    batched steps timed with CUDA events on the library's stream."""
    from dvmpp_b200 import native as N

    sims = []
    for inst in instances:
        p = sim_params(inst, steps_total, 0)
        p.precision, p.rng = N.F64, N.RNG_PHILOX
        s = ctx.sim(p, *inst["body"])
        s.set_blobs(*inst["blobs"])
        sims.append(s)
    ctx.step_batch(sims, warmup, use_graph=True)
    ctx.sync()
    ctx.mark(4)
    ctx.step_batch(sims, steps, use_graph=True)
    ctx.mark(5)
    ms = ctx.elapsed_ms(4, 5)
    for s in sims:
        s.check()
        s.close()
    return ms


def run_ours(args, dist):
    from dvmpp_b200 import native as N

    t_setup = time.perf_counter()
    instances = make_instances(args.instances, args.seed)
    ctx = N.Context(dist.local)
    sms, ccmaj, ccmin = ctx.device_info()
    steps_total = args.warmup + args.steps + args.prof_steps + args.plain_steps + args.e2e_steps + 2
    prepush = args.warmup + args.steps + args.prof_steps + args.plain_steps + 1
    sims, bodies, sparams = [], [], []
    for inst in instances:
        p = sim_params(inst, steps_total, prepush, args.e2e_steps + 1 if args.e2e_steps else 0)
        bx, bz = inst["body"]
        s = ctx.sim(p, bx, bz)
        s.set_blobs(*inst["blobs"])
        s.n_hint = p.capacity
        sims.append(s)
        bodies.append((bx, bz))
        sparams.append(p)
    rng = np.random.default_rng(1234 + dist.rank)
    for s, u in zip(sims, uniforms_for(sims, rng, prepush)):
        s.push_uniforms(u)
    setup_s = time.perf_counter() - t_setup

    # pair-kernel launch shape for this batch's class (result-invariant), and
    # for the single-simulation classes the plain path uses
    tune = None
    if not args.no_autotune:
        t0 = time.perf_counter()
        b = ctx.autotune(sims, reps=1)
        singles = set()
        for s in sims:
            c = ctx.shape_class([s])
            if c not in singles:
                singles.add(c)
                ctx.autotune([s], reps=1)
        tune = {"batch_class": b["shape_class"], "best": b["best"], "best_ms": b["best_ms"],
                "default_ms": b["default_ms"], "candidates": len(b["candidates"]),
                "single_sim_classes_tuned": len(singles),
                "tuning_s": time.perf_counter() - t0}

    # warm-up (first step eager, then graph captured and replayed)
    ctx.step_batch(sims, args.warmup, use_graph=True)
    for s in sims:
        s.check()
    ctx.sync()

    # ---- timed region: K batched steps, inputs resident in HBM, graph replay
    clocks = ClockSampler(dist.local)
    dist.barrier()
    ctx.sync()
    clocks.start()
    l0 = ctx.launches()
    ctx.profiler_range(True)  # an external profiler run with collection off sees only this
    ctx.mark(0)
    ctx.step_batch(sims, args.steps, use_graph=True)
    ctx.mark(1)
    ms = ctx.elapsed_ms(0, 1)
    ctx.profiler_range(False)
    launches = ctx.launches() - l0
    clock_info = clocks.stop()
    for s in sims:
        s.check()
    ms_max = dist.max(ms)
    value = dist.world * args.instances * args.steps / (ms_max / 1e3)

    # ---- profiled steps (eager, CUDA events around every kernel family)
    ctx.set_profiling(True)
    ctx.profile_reset()
    pairs = 0
    for _ in range(args.prof_steps):
        ns = [s.n for s in sims]
        pairs += sum(n * (n - 1) for n in ns)
        ctx.step_batch(sims, 1, use_graph=False)
    prof = ctx.profile()
    ctx.set_profiling(False)
    nb_ms, nb_n = prof["nbody"]
    step_ms_prof = prof["step"][0] / max(prof["step"][1], 1)
    nbody_launch_ms = nb_ms / max(nb_n, 1)
    pairs_per_launch = pairs / max(nb_n, 1)
    achieved_tflops = (12.0 * pairs_per_launch / (nbody_launch_ms / 1e3) / 1e12
                       if nbody_launch_ms > 0 else 0.0)  # no profiled steps: not measured
    pk = peaks()
    sm_max = float(pk.get("sm_max_mhz", 1965.0))
    fp32_peak = sms * 128 * 2 * sm_max * 1e6 / 1e12

    # ---- accuracy of the timed arithmetic: FP64 on the identical state
    accuracy = None
    if not args.no_accuracy:
        accuracy = accuracy_vs_f64(ctx, sims, bodies, sparams)

    # ---- plain GPU path: one simulation at a time, same kernels, no batching
    ctx.sync()
    ctx.mark(2)
    for _ in range(args.plain_steps):
        for s in sims:
            s.step(1)
    ctx.mark(3)
    plain_ms = ctx.elapsed_ms(2, 3)
    for s in sims:
        s.check()
    plain_ms = dist.max(plain_ms)
    plain_value = (dist.world * args.instances * args.plain_steps / (plain_ms / 1e3)
                   if args.plain_steps > 0 and plain_ms > 0 else None)

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        # The user's loop, pipelined as an application would run it: while the
        # GPU computes step k the host generates step k+1's uniforms, pushes
        # them (copy stream) and enqueues step k+1; step k's snapshot (x, z,
        # circ of every blob and the loads, taken on the GPU right after step k)
        # is then copied out while step k+1 runs.  Uniforms are pushed for an
        # upper bound of the next step's draws (the device consumes them in
        # order; the surplus carries over).
        M = 3
        ub = [2 * (s.n_hint + 2 * (M + 1) * s.np) + 2 * (M + 1) * s.np + 64 for s in sims]
        hbuf = [[pinned(u) for u in ub] for _ in range(2)]
        out_x = [pinned(s.n_hint) for s in sims]
        out_z = [pinned(s.n_hint) for s in sims]
        out_c = [pinned(s.n_hint) for s in sims]
        nprev = [s.n for s in sims]

        def generate(bufs):
            sizes = []
            for sm, hb, n in zip(sims, bufs, nprev):
                need = 2 * (n + 2 * (M + 1) * sm.np) + 2 * (M + 1) * sm.np + 64
                hb[:need] = 1.0 - rng.random(need)
                sizes.append(need)
            return sizes

        h2d = d2h = 0
        sizes = generate(hbuf[0])  # the first step's input, staged in pinned memory
        dist.barrier()
        ctx.sync()
        t0 = time.perf_counter()
        ctx.batch_push_uniforms_async(sims, hbuf[0], sizes)
        h2d += 8 * sum(sizes)
        ctx.step_batch(sims, 1, use_graph=True)
        ctx.batch_get_state_async(sims)
        for step in range(args.e2e_steps):
            last = step + 1 == args.e2e_steps
            if not last:
                sizes = generate(hbuf[(step + 1) % 2])  # overlaps the GPU step
                ctx.batch_push_uniforms_async(sims, hbuf[(step + 1) % 2], sizes)
                h2d += 8 * sum(sizes)
                ctx.step_batch(sims, 1, use_graph=True)  # queued behind this step
            # this step's x, z, circ and loads; the copy overlaps the next step
            nprev, loads = ctx.batch_wait_state(out_x, out_z, out_c)
            d2h += sum(3 * 8 * n + 4 * 8 for n in nprev)
            if not last:
                ctx.batch_get_state_async(sims)
        ctx.sync()
        e2e_s = dist.max(time.perf_counter() - t0)
        e2e = {"value": dist.world * args.instances * args.e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d / args.e2e_steps),
               "d2h_bytes_per_step": int(d2h / args.e2e_steps),
               "note": "per step: the step's uniforms (inject mode) pushed from pinned "
                       "memory, one batched step, x/z/circ of every blob and the loads "
                       "read back (what DVMBase::write_outputs consumes); pipelined: the "
                       "next step's uniforms are generated and pushed and the next step "
                       "enqueued while the GPU computes, and a step's state is copied "
                       "out while the next one runs (the first step's uniforms are "
                       "generated before the clock starts); host wall clock"}
        for s in sims:
            s.check()

    # ---- CPU baseline (rank 0, N = 1): the reference itself, bounded sample
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        r = reference_sample(instances, [0.0, 0.25, 0.5, 0.75, 1.0])
        if r:
            cpu = {"value": args.instances / r["batch_step_s"], "unit": UNIT, "cores": _cores(),
                   "kind": "reference",
                   "sample": "the instances at size quantiles 0, 0.25, 0.5, 0.75 and 1; "
                             + REF_SAMPLE_NOTE + f"; {r['wall_s']:.1f} s of CPU work",
                   "sampled": r["sampled"], "rates": r["rates"],
                   "s_per_step_by_phase": r["phases_s"]}

    nblobs = [s.n for s in sims]
    for s in sims:
        s.close()
    f64 = None
    if args.f64_steps > 0:
        f64_ms = dist.max(run_f64(ctx, instances, 3 + args.f64_steps, 1, args.f64_steps))
        f64 = {"value": dist.world * args.instances * args.f64_steps / (f64_ms / 1e3), "unit": UNIT,
               "steps": args.f64_steps, "ms_per_step": f64_ms / args.f64_steps,
               "how": "the same 64 simulations from the same initial state with every pair "
                      "sum in FP64 in the reference's operation order (the arithmetic of the "
                      "reference arm), Philox walk, graph-replayed batched steps after one "
                      "warm-up step; CUDA events"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 pair sums (Kahan), f64 state/sheet",
        "data": "synthetic (seeded bodies and wakes)",
        "config": {"workload": "batched: 64 mixed bodies (circle / ellipse aspect U[1,4] / "
                               "rounded square), panels log-U[64,512], wakes log-U[1e4,4e5] "
                               "blobs, Euler dt=0.005, nu=1e-3, ux=1, REFLECT, FP32 compensated",
                   "instances": args.instances, "blobs_total": int(sum(nblobs)),
                   "panels_total": int(sum(s.np for s in sims)),
                   "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (state + workspace >> 126 MB)",
                   "graph": "one CUDA graph per step, replayed"},
        "plain_gpu": {"value": plain_value, "unit": UNIT, "steps": args.plain_steps,
                      "ratio_batched_over_plain": value / plain_value if plain_value else None,
                      "how": "each simulation stepped alone (its own launches, no batching)"},
        "roofline": {"bound": "fp32", "kernel": "k_self_f32 (pair kernel)",
                     "achieved": achieved_tflops, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved_tflops / fp32_peak,
                     "traffic": args.traffic if args.traffic is not None else committed_traffic(),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one "
                                       "launch of this workload (profiles/"
                                       "bench_batched64_launches.md)",
                     "flops_per_pair": 12, "pairs_per_launch": pairs_per_launch,
                     "launch_ms": nbody_launch_ms,
                     "peak_source": f"derived: {sms} SMs x 128 FP32 lanes x 2 x "
                                    f"{sm_max:.0f} MHz (sm_max_mhz of MEASURED_PEAKS.json); "
                                    f"that file has no FP32 figure",
                     "share_of_step": nb_ms / max(prof["step"][0], 1e-9)},
        "profile_ms_per_step": {k: v[0] / max(args.prof_steps, 1) for k, v in prof.items()},
        "autotune": tune,
        "gpu_launches": int(launches),
        "gpu_launches_note": "own kernels in the timed region; each step's Morton sort adds "
                             "the CUB radix-sort kernels compiled into the same library "
                             "(7 per step in the ncu launch list)",
        "clocks": clock_info,
        "setup_s": setup_s,
    }
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    if accuracy:
        line["accuracy"] = accuracy
    if f64:
        line["f64_value"] = f64["value"]
        line["f64"] = f64
    ctx.close()

    # ---- the standalone N-body configuration (N = 2^20 wake) and the serving
    # loop (continuous batching vs the plain serial path): reported beside
    # (single-GPU runs only: these legs use device 0 and are not part of the
    # replicated job)
    if args.nbody_n and dist.world == 1:
        from dvmpp_b200 import cases

        nb = cases.run_nbody(args.nbody_n, [N.F32], 2)
        r = nb["results"]["f32"]
        line["nbody"] = {"n": args.nbody_n, "pair_kernel_ms": r["pair_kernel_ms"],
                         "gpairs_per_s": r["gpairs_per_s"], "tflops_12_per_pair": r["tflops_12_per_pair"],
                         "fp32_peak_frac": r["fp32_peak_frac"]}
    if args.serve_requests and dist.world == 1:
        from dvmpp_b200 import cases

        keys = ("requests", "completed", "failed", "sim_steps", "sim_steps_per_s",
                "blobs_per_panel_step",
                "latency_p50_s", "latency_p95_s", "latency_p99_s", "queue_p50_s", "queue_p99_s",
                "peak_active", "peak_bytes", "wall_s", "admit_s", "step_s", "retire_s", "ticks")
        steps = tuple(args.serve_steps)
        legs = {}
        # arrivals honoured: a feeder thread submits every request at its Poisson
        # arrival time into the running server (live intake)
        sv = cases.run_serving(args.serve_requests, 7, 20.0, steps, (64, 512), 256, 150.0,
                               True, False, live=True)
        legs["realtime_live"] = {"batched": {k: sv["batched"][k] for k in keys}}
        # throughput: every request queued at t = 0, batched vs the plain path
        sv = cases.run_serving(args.serve_requests, 7, 20.0, steps, (64, 512), 256, 150.0,
                               False, not args.no_serial)
        legs["saturated"] = {m: {k: sv[m][k] for k in keys} for m in ("batched", "serial")
                             if m in sv}
        if "speedup_sim_steps" in sv:
            legs["saturated"]["ratio_batched_over_serial"] = sv["speedup_sim_steps"]
        line["serving"] = {
            "requests": args.serve_requests,
            "arrivals": "Poisson 20 req/s (seed 7); realtime_live: each request submitted at its "
                        "arrival time by a host thread while the server runs (arrival stamped "
                        "at submission); saturated: every request queued at t = 0",
            "steps": f"U{{{steps[0]}..{steps[1]}}} (scaled from U{{100..2000}})",
            "panels": "U{64..512}", "budget_gb": 150.0, "max_active": 256,
            "bodies": "circle / ellipse / rounded square / Joukowski", **legs}
    if dist.rank == 0:
        print(json.dumps(line))
    if accuracy and not accuracy["within_bounds"]:
        sys.stderr.write("accuracy outside its bounds: " + json.dumps(accuracy["worst"]) + "\n")
        sys.exit(3)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--prof-steps", type=int, default=2)
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--f64-steps", type=int, default=2,
                    help="timed steps of the all-FP64 batch (0: skip)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the FP32-vs-FP64 check of the timed state")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in pair-kernel launch shape")
    ap.add_argument("--nbody-n", type=int, default=1 << 20,
                    help="standalone N-body leg size (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=1000,
                    help="serving leg request count (0: skip)")
    ap.add_argument("--serve-steps", type=int, nargs=2, default=[20, 100],
                    help="range of the serving requests' step counts")
    ap.add_argument("--no-serial", action="store_true",
                    help="skip the serial plain-GPU serving run")
    ap.add_argument("--traffic", type=float, default=None,
                    help="dram bytes per pair-kernel launch from an ncu capture")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference_arm(args, dist)
        else:
            run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
