"""Command-line drivers for the standalone workloads.

    python -m dvmpp_b200.cases nbody --n 1048576 [--prec f32|f64|both] [--reps 3]

nbody: the standalone regularised Biot-Savart workload -- N blobs, 70 % in a
wake x ~ U[0.5, 20], z ~ N(0, 1), 30 % in the annulus 0.5 < r < 1.5,
Gamma ~ N(0, 1e-3) summing to zero, sigma = 0.081880 (ds^0.675 of the
128-panel R = 0.5 circle), seed 2.  Prints one JSON line with the pair
kernel's CUDA-event time, pairs/s, FP32-pipe fraction and (with both
precisions) the FP32-vs-FP64 error.

    python -m dvmpp_b200.cases precision [--steps 20] [--n-wake 524288] [--panels 1024]
                                         [--eval-every 50] [--f64-steps 150]

precision: ellipse (0.5, 0.25) at 20 degrees, 1024 panels (a 1025 x 1024
influence matrix), a 2^19-blob wake, RK3 dt = 0.002; the FP32-compensated run
(FP64 QR, FP64 refinement and Kelvin row) against an all-FP64 run.

    python -m dvmpp_b200.cases sheet [--n 131072] [--panels 1024] [--reps 3]

sheet: the FP32 sheet-on-blob velocity alone (ellipse at 20 degrees, wake of
n blobs); prints its CUDA-event time, pairs/s and FP32 fraction (67 flop/pair).

    python -m dvmpp_b200.cases book [--n 4194304] [--panels 256] [--inside 0.02]

book: the Philox walk, REFLECT and DELETE alone on one simulation (CUDA events).

    python -m dvmpp_b200.cases rhs [--n 131072] [--panels 1024] [--reps 3]

rhs: the blob-on-collocation right-hand side alone (same body and wake);
prints its CUDA-event time per launch, pairs/s and FP32 fraction (12 flop/pair).

    python -m dvmpp_b200.cases serve [--requests 100] [--serial] [--realtime] [--live]

serve: the continuous-batching server on Poisson arrivals (seed 7, 20 req/s).
"""
from __future__ import annotations

import argparse
import json
import os
import time

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


def _reserve_for(ctx, reqs, max_active):
    """What a deployment configures before it opens its intake: the shared
    workspace for max_active of the largest simulations it admits, and the
    memory pool mapped for their slabs (so admissions never grow either)."""
    caps = sorted((serve_params(r).capacity for r in reqs), reverse=True)[:max_active]
    slabs = sorted((N.sim_bytes(serve_params(r), r["npanels"]) for r in reqs),
                   reverse=True)[:max_active]
    max_np = max(r["npanels"] for r in reqs)
    ctx.reserve(sum(caps), min(max_active, len(reqs)), max_np)
    ctx.pool_reserve(sum(slabs) + 8 * (3 * max_np * max_np + 64 * max_np))


def run_serving(count: int, seed: int, rate: float, steps_range, panels_range, max_active: int,
                budget_gb: float, realtime: bool, serial_too: bool, graph: bool = True,
                sync: bool = True, autotune: bool = False, live: bool = False,
                batched: bool = True, serial_every: int = 1):
    """The serving workload, continuous batching and (optionally) the plain
    serial path on the same requests; returns both summaries.

    live: the requests are not pre-submitted; a feeder thread submits each at
    its Poisson arrival time while the server runs (DVM_SERVE_LIVE), so every
    arrival is stamped by the server at submission.
    serial_every: the serial path runs every k-th request only (its sim-steps/s
    is then a rate on a sample of the same distribution)."""
    import threading

    all_reqs = W.serving_requests(count, seed, rate, steps_range, panels_range)
    out = {"workload": "serving", "requests": count, "rate_per_s": rate,
           "steps_range": list(steps_range), "panels_range": list(panels_range),
           "budget_gb": budget_gb, "realtime": realtime, "live_intake": live,
           "serial_every": serial_every}
    modes = ([("batched", False)] if batched else []) + ([("serial", True)] if serial_too else [])
    for name, serial in modes:
        reqs = all_reqs[::serial_every] if serial else all_reqs
        ctx = N.Context(0)
        srv = N.Server(ctx, budget_bytes=int(budget_gb * 2**30), max_active=max_active)
        srv.set_option(N.SERVE_GRAPH, 1 if graph else 0)
        srv.set_option(N.SERVE_SYNC, 1 if sync else 0)
        srv.set_option(N.SERVE_AUTOTUNE, 1 if autotune else 0)
        if live:
            _reserve_for(ctx, reqs, 1 if serial else max_active)
            srv.set_option(N.SERVE_LIVE, 1)
            errors = []

            def feed():
                try:
                    t0 = time.perf_counter()
                    for r in reqs:
                        wait = r["arrival"] - (time.perf_counter() - t0)
                        if wait > 0:
                            time.sleep(wait)
                        srv.submit(serve_params(r), *r["body"], r["steps"])
                except Exception as e:  # reported below
                    errors.append(e)
                finally:
                    srv.close_intake()

            feeder = threading.Thread(target=feed)
            feeder.start()
            srv.run(serial=serial, realtime=True)
            feeder.join()
            if errors:
                raise errors[0]
        else:
            for r in reqs:
                srv.submit(serve_params(r), *r["body"], r["steps"], r["arrival"])
            srv.run(serial=serial, realtime=realtime)
        out[name] = srv.stats()
        # blob growth: blobs at the end per (panel x step) over the completed
        # requests (each starts empty), for extrapolating to other step ranges
        nb = npsteps = 0
        for rid in range(out[name]["requests"]):
            res = srv.result(rid)
            if res["status"] == 0 and res["steps_done"] > 0:
                nb += res["blobs"]
                npsteps += reqs[rid]["npanels"] * res["steps_done"]
        out[name]["blobs_per_panel_step"] = nb / npsteps if npsteps else None
        srv.close()
        ctx.close()
    if serial_too and batched:
        out["speedup_sim_steps"] = (out["batched"]["sim_steps_per_s"]
                                    / max(out["serial"]["sim_steps_per_s"], 1e-12))
    return out


def _evaluate(sim):
    """Fields, panel strengths, right-hand side and loads of a simulation's
    current state without moving it (biotsavart, solvevortexsheet,
    vortexsheetbc, compute_loads)."""
    for ph in (N.PHASE_BIOTSAVART, N.PHASE_SOLVE, N.PHASE_SHEETBC, N.PHASE_LOADS):
        sim.phase(ph)
    return sim.blobs(), sim.gamma(), sim.rhs(), sim.loads()


def _same_state_errors(ctx, sim32, params64, body):
    """The FP32 simulation's current state evaluated in place and by an FP64
    copy of it (same body, capacity and parameters): rel-L2 and max-norm
    errors of u, w, uvs, wvs, gamma and the right-hand side; Cd / Cl errors."""
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    mx = lambda a, b: float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    d32, g32, b32, l32 = _evaluate(sim32)
    ref = ctx.sim(params64, *body)
    ref.set_blobs(d32["x"], d32["z"], d32["circ"], d32["sigma"])
    dd, gd, bd, ld = _evaluate(ref)
    ref.close()
    out = {"n": int(dd["x"].size), "gamma_rel_l2": rel(g32, gd), "gamma_max": mx(g32, gd),
           "rhs_rel_l2": rel(b32[:-1], bd[:-1]), "rhs_max": mx(b32[:-1], bd[:-1]),
           "kelvin_row_abs": float(abs(b32[-1] - bd[-1]))}
    for key in ("u", "w", "uvs", "wvs"):
        out[key + "_rel_l2"] = rel(d32[key], dd[key])
        out[key + "_max"] = mx(d32[key], dd[key])
    cmag = float(np.hypot(ld[2], ld[3]))
    out.update({"cd_f32": l32[2], "cd_f64": ld[2], "cl_f32": l32[3], "cl_f64": ld[3],
                "cd_err_of_force": abs(l32[2] - ld[2]) / cmag if cmag > 0 else 0.0,
                "cl_err_of_force": abs(l32[3] - ld[3]) / cmag if cmag > 0 else 0.0})
    return out


def run_precision(steps: int, n_wake: int, npanels: int = 1024, seed: int = 2,
                  incidence_deg: float = 20.0, eval_every: int = 0, f64_steps=None):
    """Sheet-solve precision: an ellipse (semi-axes 0.5, 0.25) at the given
    incidence, npanels panels, a wake of n_wake blobs (the N-body distribution,
    core size ds^0.675 of this body), RK3 with dt = 0.002, nu = 1e-3, ux = 1.
    One run with FP32 compensated pair sums (FP64 QR + FP64 refinement,
    Kelvin row in FP64) for `steps` steps beside an all-FP64 run from the same
    state and the same Philox stream for the first `f64_steps` of them (all by
    default).  Reports per-step gamma / Cd / Cl differences while both run,
    the blob counts, the least-squares solvers against each other on one
    right-hand side, and -- every `eval_every` steps and at the end -- the
    FP32 run's state evaluated in both arithmetics (fields, gamma, RHS,
    Cd / Cl on the identical state)."""
    M = 3
    f64_steps = steps if f64_steps is None else min(f64_steps, steps)
    ctx = N.Context(0)
    bx, bz = W.ellipse(npanels, 0.5, 0.25, incidence_deg)
    ds = np.hypot(np.diff(bx), np.diff(bz))
    sigma = float(np.mean(ds)) ** 0.675
    x, z, g, s = W.wake(n_wake, seed, sigma)
    cap = n_wake + (steps + 2) * (M + 1) * npanels + 4096
    common = dict(rho=1.0, nu=1e-3, dt=0.002, ux=1.0, uz=0.0, max_numpanelvort=M,
                  scheme=N.RK3, surface_cross=N.REFLECT, rng=N.RNG_PHILOX, seed=11,
                  capacity=cap)
    p64 = N.Params(precision=N.F64, **common)
    sims = {name: ctx.sim(N.Params(precision=prec, **common), bx, bz)
            for name, prec in (("f32", N.F32), ("f64", N.F64))}
    for sim in sims.values():
        sim.set_blobs(x, z, g, s)
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    # least-squares solvers on one right-hand side (the initial wake's)
    s64 = sims["f64"]
    s64.phase(N.PHASE_SOLVE)
    A, b, g_qr = s64.influence(), s64.rhs(), s64.gamma()
    g_ls = np.linalg.lstsq(A, b, rcond=None)[0]
    g_ne = np.linalg.solve(A.T @ A, A.T @ b)
    sims["f32"].phase(N.PHASE_SOLVE)
    solve = {"matrix": list(A.shape), "cond_A": float(np.linalg.cond(A)),
             "qr_refined_vs_lstsq": rel(g_qr, g_ls),
             "normal_equations_vs_lstsq": rel(g_ne, g_ls),
             "f32_rhs_qr_refined_vs_f64": rel(sims["f32"].gamma(), g_qr),
             "residual_norm_qr": float(np.linalg.norm(A @ g_qr - b)),
             "residual_norm_lstsq": float(np.linalg.norm(A @ g_ls - b))}

    rows, checkpoints = [], []
    t = {"f32": 0.0, "f64": 0.0}
    for k in range(steps):
        active = ("f32", "f64") if k < f64_steps else ("f32",)
        for name in active:
            sim = sims[name]
            ctx.sync()
            t0 = time.perf_counter()
            sim.step(1)
            ctx.sync()
            t[name] += time.perf_counter() - t0
            sim.check()
        if k < f64_steps:
            l32, l64 = sims["f32"].loads(), sims["f64"].loads()
            rows.append({"step": k + 1, "n_f32": sims["f32"].n, "n_f64": sims["f64"].n,
                         "gamma_rel_l2": rel(sims["f32"].gamma(), sims["f64"].gamma()),
                         "cd_f32": l32[2], "cd_f64": l64[2], "cl_f32": l32[3], "cl_f64": l64[3]})
        if eval_every and ((k + 1) % eval_every == 0 or k + 1 == steps):
            cp = _same_state_errors(ctx, sims["f32"], p64, (bx, bz))
            cp["step"] = k + 1
            checkpoints.append(cp)

    # both precisions evaluated on one identical state (the FP64 run's last one)
    d64 = sims["f64"].blobs()
    sims["f32"].set_blobs(d64["x"], d64["z"], d64["circ"], d64["sigma"])
    fields = {}
    for name, sim in sims.items():
        for ph in (N.PHASE_BIOTSAVART, N.PHASE_SOLVE, N.PHASE_SHEETBC):
            sim.phase(ph)
        d = sim.blobs()
        fields[name] = (d, sim.gamma(), sim.rhs())
    (d32, g32, b32), (dd, gd, bd) = fields["f32"], fields["f64"]
    mx = lambda a, b: float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    same_state = {"n": int(dd["x"].size), "gamma_rel_l2": rel(g32, gd), "gamma_max": mx(g32, gd),
                  "rhs_rel_l2": rel(b32[:-1], bd[:-1]), "rhs_max": mx(b32[:-1], bd[:-1]),
                  "kelvin_row_abs": float(abs(b32[-1] - bd[-1]))}
    for key in ("u", "w", "uvs", "wvs"):
        same_state[key + "_rel_l2"] = rel(d32[key], dd[key])
        same_state[key + "_max"] = mx(d32[key], dd[key])
    # the FP32 sheet-on-blob kernel alone: both evaluate with the FP64 gamma
    sims["f32"].set_gamma(gd)
    sims["f32"].phase(N.PHASE_SHEETBC)
    ds32 = sims["f32"].blobs()
    for key in ("uvs", "wvs"):
        same_state[key + "_same_gamma_rel_l2"] = rel(ds32[key], dd[key])
        same_state[key + "_same_gamma_max"] = mx(ds32[key], dd[key])
    ctx.close()
    cd_err = max((abs(r["cd_f32"] - r["cd_f64"]) / max(abs(r["cd_f64"]), 1e-12) for r in rows),
                 default=0.0)
    cl_err = max((abs(r["cl_f32"] - r["cl_f64"]) for r in rows), default=0.0)
    force = [float(np.hypot(r["cd_f64"], r["cl_f64"])) for r in rows]
    cd_f = max((abs(r["cd_f32"] - r["cd_f64"]) / f for r, f in zip(rows, force) if f > 0), default=0.0)
    cl_f = max((abs(r["cl_f32"] - r["cl_f64"]) / f for r, f in zip(rows, force) if f > 0), default=0.0)
    return {"workload": "precision", "npanels": npanels, "incidence_deg": incidence_deg,
            "n_wake": n_wake, "sigma": sigma, "steps": steps, "f64_steps": f64_steps,
            "scheme": "RK3", "dt": 0.002, "solve": solve, "same_state": same_state,
            "checkpoints": checkpoints,
            "run": {"steps_with_equal_n": sum(r["n_f32"] == r["n_f64"] for r in rows),
                    "max_gamma_rel_l2": max((r["gamma_rel_l2"] for r in rows), default=0.0),
                    "max_cd_rel": cd_err, "max_cl_abs": cl_err,
                    "max_cd_err_of_force": cd_f, "max_cl_err_of_force": cl_f,
                    "final": rows[-1] if rows else None,
                    "n_f32_final": sims_n_final(checkpoints, rows),
                    "s_per_step_f32": t["f32"] / max(steps, 1),
                    "s_per_step_f64": t["f64"] / max(f64_steps, 1)},
            "per_step": rows}


def sims_n_final(checkpoints, rows):
    if checkpoints:
        return checkpoints[-1]["n"]
    return rows[-1]["n_f32"] if rows else None


def run_sheet(n: int, npanels: int, reps: int, seed: int = 2):
    """Sheet-on-blob velocity alone: an ellipse (0.5, 0.25) at 20 degrees with
    npanels panels, an n-blob wake (the N-body distribution, core size of this
    body), FP32 instance; blob velocities and the panel strengths are computed
    once, then the sheet-on-blob phase runs reps times (the first untimed)."""
    ctx = N.Context(0)
    sms, _, _ = ctx.device_info()
    bx, bz = W.ellipse(npanels, incidence_deg=20.0)
    x, z, g, s = W.wake(n, seed, W.core_size(bx, bz))
    sim = ctx.sim(N.Params(capacity=n, precision=N.F32, rng=N.RNG_PHILOX, ux=1.0), bx, bz)
    sim.set_blobs(x, z, g, s)
    sim.phase(N.PHASE_BIOTSAVART)
    sim.phase(N.PHASE_SOLVE)
    sim.phase(N.PHASE_SHEETBC)  # warm-up
    ctx.mark(0)  # CUDA events on the library's stream around the timed launches
    for _ in range(reps):
        sim.phase(N.PHASE_SHEETBC)
    ctx.mark(1)
    ms = ctx.elapsed_ms(0, 1) / max(reps, 1)
    pairs = n * npanels
    tf = 67.0 * pairs / (ms / 1e3) / 1e12
    sim.close()
    ctx.close()
    return {"workload": "sheet", "n": n, "panels": npanels, "pairs": pairs, "kernel_ms": ms,
            "gpairs_per_s": pairs / (ms / 1e3) / 1e9, "tflops_67_per_pair": tf,
            "fp32_peak_frac": tf / _fp32_peak_tflops(sms)}


def run_rhs(n: int, npanels: int, reps: int, seed: int = 2):
    """Blob-on-collocation right-hand side alone (the at-target kernel of
    solvevortexsheet, src/VortexSheet.cpp:181-203): an ellipse (0.5, 0.25) at
    20 degrees with npanels panels and an n-blob wake, FP32 instance; the
    profiled RHS family's CUDA-event time per launch, pairs/s and the FP32
    fraction at 12 flop per pair."""
    ctx = N.Context(0)
    sms, _, _ = ctx.device_info()
    bx, bz = W.ellipse(npanels, incidence_deg=20.0)
    x, z, g, s = W.wake(n, seed, W.core_size(bx, bz))
    sim = ctx.sim(N.Params(capacity=n + 8 * npanels, precision=N.F32, rng=N.RNG_PHILOX, ux=1.0),
                  bx, bz)
    sim.set_blobs(x, z, g, s)
    sim.step(1)  # warm-up: one whole step (the batched RHS launch included)
    sim.set_blobs(x, z, g, s)
    ctx.set_profiling(True)
    ctx.profile_reset()
    for _ in range(reps):
        sim.step(1)
        sim.set_blobs(x, z, g, s)
    prof = ctx.profile()
    ctx.set_profiling(False)
    ms = prof["rhs"][0] / max(prof["rhs"][1], 1)
    pairs = n * npanels
    tf = 12.0 * pairs / (ms / 1e3) / 1e12
    sim.close()
    ctx.close()
    return {"workload": "rhs", "n": n, "panels": npanels, "pairs": pairs, "kernel_ms": ms,
            "gpairs_per_s": pairs / (ms / 1e3) / 1e9, "tflops_12_per_pair": tf,
            "fp32_peak_frac": tf / _fp32_peak_tflops(sms)}


def run_setup(panels=(64, 128, 256, 512, 1024), reps: int = 5):
    """Per-body set-up (src/VortexSheet.cpp:78-165 plus the factorisation that
    replaces the per-step LAPACK solve): wall time of creating a simulation on a
    circle of np panels -- geometry, uploads, influence matrix, QR, P -- best of
    `reps` after one warm-up creation."""
    import time
    ctx = N.Context(0)
    out = {"workload": "setup", "reps": reps, "ms": {}}
    for npan in panels:
        bx, bz = W.circle(npan)
        ctx.sim(N.Params(capacity=1024), bx, bz).close()
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            sim = ctx.sim(N.Params(capacity=1024), bx, bz)
            ctx.sync()
            best = min(best, time.perf_counter() - t0)
            sim.close()
        out["ms"][str(npan)] = best * 1e3
    ctx.close()
    return out


def run_book(n: int, npanels: int, inside: float, reps: int, seed: int = 3):
    """Bookkeeping phases alone on one simulation: a circle of npanels panels
    (R = 0.5) and n blobs, a fraction `inside` of them inside the body, the rest
    in the wake distribution.  CUDA-event time per call of the Philox random
    walk, REFLECT and DELETE (the blob state is restored between calls), with
    the algorithmic bytes per blob: walk 32 (read and write x, z), crossing
    flags 17 (read x, z; a flag), DELETE's move 132 per kept blob (read x, z
    and the other six arrays, write all eight and the ID)."""
    ctx = N.Context(0)
    bx, bz = W.circle(npanels)
    x, z, g, s = W.wake(n, seed, W.core_size(bx, bz))
    rng = np.random.default_rng(seed)
    k = rng.random(n) < inside
    r = 0.45 * np.sqrt(rng.random(int(k.sum())))
    th = rng.uniform(0, 2 * np.pi, r.size)
    x[k], z[k] = r * np.cos(th), r * np.sin(th)
    out = {"workload": "bookkeeping", "n": n, "panels": npanels, "inside": inside}
    for name, cross, phase in (("walk_philox", N.REFLECT, N.PHASE_DIFFUSE),
                               ("reflect", N.REFLECT, N.PHASE_REFLECT),
                               ("delete", N.DELETE, N.PHASE_DELETE)):
        sim = ctx.sim(N.Params(capacity=n, rng=N.RNG_PHILOX, surface_cross=cross), bx, bz)
        ms = []
        for rep in range(reps + 1):
            sim.set_blobs(x, z, g, s)
            ctx.mark(0)
            sim.phase(phase)
            ctx.mark(1)
            if rep:
                ms.append(ctx.elapsed_ms(0, 1))
        sim.check()
        out[name + "_ms"] = float(np.median(ms))
        if name == "delete":
            kept = sim.n
            out["delete_kept"] = kept
            out["delete_gbs_algorithmic"] = (17.0 * n + 132.0 * kept) / (out[name + "_ms"] / 1e3) / 1e9
        sim.close()
    out["walk_gbs_algorithmic"] = 32.0 * n / (out["walk_philox_ms"] / 1e3) / 1e9
    ctx.close()
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
    sv.add_argument("--autotune", action="store_true",
                    help="tune the pair kernel once per new batch-shape class")
    sv.add_argument("--live", action="store_true",
                    help="submit each request at its arrival time while the server runs")
    sv.add_argument("--serial-every", type=int, default=1,
                    help="the serial path runs every k-th request only")
    sh = sub.add_parser("sheet")
    sh.add_argument("--n", type=int, default=1 << 17)
    sh.add_argument("--panels", type=int, default=1024)
    sh.add_argument("--reps", type=int, default=3)
    bk = sub.add_parser("book")
    bk.add_argument("--n", type=int, default=1 << 22)
    bk.add_argument("--panels", type=int, default=256)
    bk.add_argument("--inside", type=float, default=0.02)
    bk.add_argument("--reps", type=int, default=5)
    rh = sub.add_parser("rhs")
    rh.add_argument("--n", type=int, default=1 << 17)
    rh.add_argument("--panels", type=int, default=1024)
    rh.add_argument("--reps", type=int, default=3)
    su = sub.add_parser("setup")
    su.add_argument("--reps", type=int, default=5)
    pr = sub.add_parser("precision")
    pr.add_argument("--steps", type=int, default=20)
    pr.add_argument("--n-wake", type=int, default=1 << 19)
    pr.add_argument("--panels", type=int, default=1024)
    pr.add_argument("--seed", type=int, default=2)
    pr.add_argument("--eval-every", type=int, default=0,
                    help="evaluate the FP32 run's state in FP64 every this many steps")
    pr.add_argument("--f64-steps", type=int, default=None,
                    help="carry the all-FP64 run this many steps (default: all)")
    a = ap.parse_args(argv)
    if a.cmd == "precision":
        print(json.dumps(run_precision(a.steps, a.n_wake, a.panels, a.seed,
                                       eval_every=a.eval_every, f64_steps=a.f64_steps)))
    if a.cmd == "serve":
        print(json.dumps(run_serving(a.requests, a.seed, a.rate, tuple(a.steps), tuple(a.panels),
                                     a.max_active, a.budget_gb, a.realtime or a.live, a.serial,
                                     not a.no_graph, not a.no_sync, a.autotune, a.live,
                                     serial_every=a.serial_every)))
    if a.cmd == "setup":
        print(json.dumps(run_setup(reps=a.reps)))
    if a.cmd == "sheet":
        print(json.dumps(run_sheet(a.n, a.panels, a.reps)))
    if a.cmd == "book":
        print(json.dumps(run_book(a.n, a.panels, a.inside, a.reps)))
    if a.cmd == "rhs":
        print(json.dumps(run_rhs(a.n, a.panels, a.reps)))
    if a.cmd == "nbody":
        precs = {"f32": [N.F32], "f64": [N.F64], "both": [N.F32, N.F64]}[a.prec]
        print(json.dumps(run_nbody(a.n, precs, a.reps, a.seed)))


if __name__ == "__main__":
    main()
