"""Plain-DVM cylinder run on the GPU against the CPU oracle, step by step.

Configuration (the reference's plain DVM case): circular cylinder R = 0.5 as a
closed contour of 129 points (128 panels), ux = 3, uz = 0, nu = 1e-3,
density 1, Euler, dt = 0.005, 150 steps, max_NumPanelVort = 3,
cutoff_exp = 0.675, REFLECT, seed 1.  The GPU runs in inject mode on the
reference's own mt19937 stream, so both sides see the same random walk.

    python tests/parity_cylinder.py [--steps 150] [--prec f64|f32]

prints one JSON line per step (N, errors of u, w, uvs, wvs, gamma, Cd, Cl) and
a summary.  Test infrastructure: it imports the oracle.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dvmpp_b200 import native as N  # noqa: E402
from dvmpp_b200 import workloads as W  # noqa: E402
from oracle.pyoracle import Port, SimParams  # noqa: E402


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


def run(steps=150, prec=N.F64, ctx=None, port=None, callback=None):
    own = ctx is None
    ctx = ctx or N.Context(0)
    port = port or Port()
    bx, bz = W.circle(128)
    p = N.Params(rho=1.0, nu=1e-3, dt=0.005, ux=3.0, uz=0.0, cutoff_exp=0.675,
                 max_numpanelvort=3, scheme=N.EULER, surface_cross=N.REFLECT, rng=N.RNG_INJECT,
                 precision=prec, seed=1, capacity=steps * 2 * 4 * 128 + 4096,
                 rng_capacity=1 << 23)
    sim = ctx.sim(p, bx, bz)
    o = port.sim(SimParams(rho=1.0, nu=1e-3, dt=0.005, ux=3.0, uz=0.0, cutoff_exp=0.675,
                           max_numpanelvort=3, scheme="euler", surface_cross="REFLECT", seed=1,
                           steps=steps), bx, bz)
    stream = port.mt_stream(1, 1 << 23)
    sim.push_uniforms(stream)
    rows = []
    area = 1.0
    den = 0.5 * 1.0 * area * 9.0  # 0.5 rho A U^2 with A = 1 (diameter), U = 3
    for k in range(1, steps + 1):
        sim.step(1)
        sim.check()
        o.step(1)
        d, e = sim.blobs(), o.blobs()
        fx, fz, cd, cl = sim.loads()
        fx0, fz0, _ = o.forces()
        row = {"step": k, "n_gpu": sim.n, "n_ref": o.n}
        if sim.n == o.n:
            for key in ("x", "z", "u", "w", "uvs", "wvs"):
                row["rel_l2_" + key] = rel_l2(d[key], e[key])
            row["max_abs_x"] = float(np.max(np.abs(d["x"] - e["x"]))) if sim.n else 0.0
        row["rel_l2_gamma"] = rel_l2(sim.gamma(), o.gamma())
        row["cd"], row["cd_ref"] = cd, fx0 / den
        row["cl"], row["cl_ref"] = cl, fz0 / den
        row["cd_rel"] = abs(cd - fx0 / den) / max(abs(fx0 / den), 1e-300)
        row["cl_abs"] = abs(cl - fz0 / den)
        rows.append(row)
        if callback:
            callback(row)
    sim.close()
    if own:
        ctx.close()
    return rows


def summary(rows):
    same_n = [r for r in rows if r["n_gpu"] == r["n_ref"]]
    out = {"steps": len(rows), "steps_with_equal_n": len(same_n),
           "first_n_mismatch": next((r["step"] for r in rows if r["n_gpu"] != r["n_ref"]), None),
           "final_n": rows[-1]["n_gpu"], "final_n_ref": rows[-1]["n_ref"],
           "max_cd_rel": max(r["cd_rel"] for r in rows),
           "max_cl_abs": max(r["cl_abs"] for r in rows),
           "max_rel_l2_gamma": max(r["rel_l2_gamma"] for r in rows)}
    for key in ("u", "w", "uvs", "wvs", "x"):
        vals = [r["rel_l2_" + key] for r in same_n if "rel_l2_" + key in r]
        out["max_rel_l2_" + key] = max(vals) if vals else None
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--prec", choices=["f64", "f32"], default="f64")
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args()
    cb = None if a.quiet else (lambda r: print(json.dumps(r), flush=True))
    rows = run(a.steps, N.F64 if a.prec == "f64" else N.F32, callback=cb)
    print(json.dumps({"summary": summary(rows), "prec": a.prec}))


if __name__ == "__main__":
    main()
