"""The standalone N-body and sheet-solve workloads at their full sizes, as parity tests.

Config 2 (standalone N-body, N = 2^20 wake + 256 collocation targets):
DirectKernel::computeSelfInduced / computeInducedAt
(src/VelocityKernel.cpp:30-109).  The FP32-compensated field against the FP64
GPU field over all 2^20 targets (rel-L2 <= 1e-5, max-norm reported), the FP64
GPU field against the CPU oracle on a 4096-target sample (<= 1e-12 of the
field's scale), and the 256 collocation targets through the at-target kernel
(FP64 <= 1e-12, FP32 rel-L2 <= 1e-5 against the oracle).

Config 3 (ellipse 0.5 x 0.25 at 20 degrees, 1024 panels, a 2^19-blob wake,
RK3, dt 0.002, nu 1e-3, ux 1): one RK3 step (src/DVMBase.cpp:182-207) of the
FP32 path and of the all-FP64 path from one identical state -- the fields,
panel strengths and right-hand side on that state within rel-L2 1e-5, equal
blob counts after the step, the step's displacements within rel-L2 1e-5 and
Cd / Cl within 0.5 % of |(Cd, Cl)|.
"""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu

SIGMA_CYL128 = 0.08188040878164335  # ds^0.675 of the 128-panel R = 0.5 circle
F64_TOL = 1e-12
F32_REL_L2 = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _self_field(ctx, x, z, g, s, prec):
    bx, bz = W.circle(128)
    sim = ctx.sim(N.Params(capacity=x.size, precision=prec, rng=N.RNG_PHILOX), bx, bz)
    sim.set_blobs(x, z, g, s)
    sim.phase(N.PHASE_BIOTSAVART)
    d = sim.blobs()
    sim.close()
    return d["u"], d["w"]


def test_config2_nbody_2pow20(ctx, port):
    n = 1 << 20
    x, z, g, s = W.wake(n, 2, SIGMA_CYL128)
    u32, w32 = _self_field(ctx, x, z, g, s, N.F32)
    u64, w64 = _self_field(ctx, x, z, g, s, N.F64)
    assert np.all(np.isfinite(u32)) and np.all(np.isfinite(w32))
    e = {"u_rel_l2": rel_l2(u32, u64), "w_rel_l2": rel_l2(w32, w64),
         "u_max": float(np.max(np.abs(u32 - u64)) / np.max(np.abs(u64))),
         "w_max": float(np.max(np.abs(w32 - w64)) / np.max(np.abs(w64)))}
    print("config 2 FP32 vs FP64:", e)
    assert e["u_rel_l2"] <= F32_REL_L2 and e["w_rel_l2"] <= F32_REL_L2, e

    # FP64 GPU against the CPU oracle on 4096 targets (computeInducedAt's
    # r^2 <= 1e-15 skip removes the self pair, as the index test does)
    pick = np.sort(np.random.default_rng(3).choice(n, 4096, replace=False))
    uo, wo = port.direct_at(x, z, g, s, x[pick], z[pick])
    sc = max(np.max(np.abs(uo)), np.max(np.abs(wo)))
    err = max(np.max(np.abs(u64[pick] - uo)), np.max(np.abs(w64[pick] - wo))) / sc
    print("config 2 FP64 GPU vs oracle (4096 targets): max rel", err)
    assert err <= F64_TOL

    # the 256 collocation targets
    tx, tz = W.collocation_circle(256)
    uo, wo = port.direct_at(x, z, g, s, tx, tz)
    sc = max(np.max(np.abs(uo)), np.max(np.abs(wo)))
    u, w = ctx.biot_savart_at(x, z, g, s, tx, tz, N.F64)
    assert max(np.max(np.abs(u - uo)), np.max(np.abs(w - wo))) <= F64_TOL * sc
    u, w = ctx.biot_savart_at(x, z, g, s, tx, tz, N.F32)
    assert rel_l2(u, uo) <= F32_REL_L2 and rel_l2(w, wo) <= F32_REL_L2


def _evaluate(sim):
    for ph in (N.PHASE_BIOTSAVART, N.PHASE_SOLVE, N.PHASE_SHEETBC, N.PHASE_LOADS):
        sim.phase(ph)
    return sim.blobs(), sim.gamma(), sim.rhs(), sim.loads()


def test_config3_full_size_rk3_step(ctx):
    npan, n_wake = 1024, 1 << 19
    bx, bz = W.ellipse(npan, 0.5, 0.25, 20.0)
    x, z, g, s = W.wake(n_wake, 2, W.core_size(bx, bz))
    common = dict(rho=1.0, nu=1e-3, dt=0.002, ux=1.0, uz=0.0, max_numpanelvort=3,
                  scheme=N.RK3, surface_cross=N.REFLECT, rng=N.RNG_PHILOX, seed=11,
                  capacity=n_wake + 16 * npan)
    sims = {p: ctx.sim(N.Params(precision=p, **common), bx, bz) for p in (N.F32, N.F64)}
    for sim in sims.values():
        sim.set_blobs(x, z, g, s)
    # the identical state, both arithmetics
    (d32, g32, b32, l32), (d64, g64, b64, l64) = (_evaluate(sims[p]) for p in (N.F32, N.F64))
    errs = {k: rel_l2(d32[k], d64[k]) for k in ("u", "w", "uvs", "wvs")}
    errs["gamma"] = rel_l2(g32, g64)
    errs["rhs"] = rel_l2(b32[:-1], b64[:-1])
    print("config 3 identical state, rel-L2:", errs)
    assert all(v <= F32_REL_L2 for v in errs.values()), errs
    # one RK3 step from that state
    for sim in sims.values():
        sim.step(1)
        sim.check()
    a32, a64 = sims[N.F32].blobs(), sims[N.F64].blobs()
    assert a32["x"].size == a64["x"].size > n_wake
    dx32 = np.concatenate([a32["x"][:n_wake] - x, a32["z"][:n_wake] - z])
    dx64 = np.concatenate([a64["x"][:n_wake] - x, a64["z"][:n_wake] - z])
    disp = rel_l2(dx32, dx64)
    f32l, f64l = sims[N.F32].loads(), sims[N.F64].loads()
    cmag = np.hypot(f64l[2], f64l[3])
    print("config 3 after one RK3 step: displacement rel-L2", disp, "loads", f32l, f64l)
    assert disp <= F32_REL_L2
    assert abs(f32l[2] - f64l[2]) <= 5e-3 * cmag and abs(f32l[3] - f64l[3]) <= 5e-3 * cmag
    assert rel_l2(sims[N.F32].gamma(), sims[N.F64].gamma()) <= F32_REL_L2
    for sim in sims.values():
        sim.close()
