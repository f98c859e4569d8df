"""Vortex-sheet, bookkeeping and whole-step parity on the GPU (C ABI).

Oracle: oracle/dvm_oracle.c, itself bit-identical to the reference sources
(tests/test_oracle_vs_ref.py).  Each phase is fed IDENTICAL inputs on both
sides; integer results (blob counts, inside flags, IDs) must be equal, FP64
results agree to the stated tolerances:
  * influence matrix, sheet-on-blob, positions: 1e-12 relative to the field's scale
  * gamma: the GPU solves the same least-squares problem by QR + refinement
    where the reference uses the normal equations; 1e-9 relative
  * forces: 1e-9 relative
"""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W
from oracle.pyoracle import SimParams

pytestmark = pytest.mark.gpu


def params(**kw):
    p = N.Params(capacity=kw.pop("capacity", 1 << 17), rng_capacity=kw.pop("rng_capacity", 1 << 22))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def oparams(p: N.Params, steps=10):
    return SimParams(rho=p.rho, nu=p.nu, dt=p.dt, ux=p.ux, uz=p.uz, cutoff_exp=p.cutoff_exp,
                     max_numpanelvort=p.max_numpanelvort,
                     scheme="euler" if p.scheme == N.EULER else "RK3",
                     surface_cross={0: "DELETE", 1: "ABSORB", 2: "REFLECT"}[p.surface_cross],
                     seed=p.seed, steps=steps)


def close(a, b, rel):
    sc = max(np.max(np.abs(b)), 1e-300) if np.size(b) else 1.0
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) <= rel * sc if np.size(b) else True


def test_geometry_and_influence_matrix(ctx, port):
    for npan in (20, 128, 1024):
        bx, bz = W.circle(npan) if npan != 1024 else W.ellipse(1024, 0.5, 0.25, 20.0)
        s = ctx.sim(params(), bx, bz)
        geo = port.sheet_geometry(bx, bz)
        pan = s.panels()
        for k in ("xc", "zc", "ds", "theta", "enx", "enz"):
            assert np.array_equal(pan[k], geo[k]), k
        A0 = port.influence_matrix(bx, bz)
        A = s.influence()
        assert A.shape == A0.shape
        assert close(A, A0, 1e-12)
        s.close()


def _random_state(n, seed, bx, bz):
    x, z, g, sg = W.wake(n, seed, W.core_size(bx, bz))
    return x, z, g, sg


@pytest.mark.parametrize("prec", [N.F64, N.F32])
def test_sheet_solve_and_velocity(ctx, port, prec):
    bx, bz = W.circle(128)
    p = params(precision=prec)
    s = ctx.sim(p, bx, bz)
    x, z, g, sg = _random_state(3000, 11, bx, bz)
    s.set_blobs(x, z, g, sg)
    geo = port.sheet_geometry(bx, bz)
    b0 = port.sheet_rhs(geo, p.ux, p.uz, x, z, g, sg)
    A0 = port.influence_matrix(bx, bz)
    g0 = port.sheet_solve(A0, b0)
    s.phase(N.PHASE_SOLVE)
    b = s.rhs()
    assert close(b, b0, 1e-12 if prec == N.F64 else 2e-6)
    gam = s.gamma()
    assert close(gam, g0, 1e-9 if prec == N.F64 else 5e-5)
    # sheet-on-blob from the oracle's gamma on both sides (FP32 instances
    # evaluate the panel terms in single precision: max error <= 1e-5 of max)
    s.set_gamma(g0)
    s.phase(N.PHASE_SHEETBC)
    uvs0, wvs0 = port.sheet_on_blobs(geo, g0, x, z)
    d = s.blobs()
    tol = 1e-12 if prec == N.F64 else 1e-5
    assert close(d["uvs"], uvs0, tol) and close(d["wvs"], wvs0, tol)
    s.close()


def test_empty_blob_solve(ctx, port):
    bx, bz = W.circle(64)
    s = ctx.sim(params(), bx, bz)
    s.phase(N.PHASE_SOLVE)
    geo = port.sheet_geometry(bx, bz)
    b0 = port.sheet_rhs(geo, 3.0, 0.0, [], [], [], [])
    assert close(s.rhs(), b0, 1e-15)
    assert close(s.gamma(), port.sheet_solve(port.influence_matrix(bx, bz), b0), 1e-9)
    s.close()


@pytest.mark.parametrize("npanels", [13, 40, 300, 700, 1100])
def test_pseudo_inverse_every_kernel_path(ctx, npanels):
    """The once-per-body factorisation has a register-resident path per column
    length (m = np + 1 <= 288, 544, 1056) and a general path above that; each
    must give the least-squares gamma of the influence matrix it built."""
    bx, bz = W.ellipse(npanels, incidence_deg=20.0)
    s = ctx.sim(params(capacity=4096, ux=1.0), bx, bz)
    s.phase(N.PHASE_SOLVE)
    A, b = s.influence(), s.rhs()
    ref = np.linalg.lstsq(A, b, rcond=None)[0]
    assert close(s.gamma(), ref, 1e-10), npanels
    s.close()


def test_group_created_sims_equal_alone(ctx):
    """dvm_sims_create factorises the bodies of a group together (up to 8 per
    cooperative launch per register class, the general path one by one); every
    simulation's saved state, which holds A and P, must equal byte for byte the
    same body created alone.  The group spans all three register classes,
    more than 8 bodies of one class, and the general path (np = 1100)."""
    panels = [13, 40, 64, 100, 150, 200, 250, 287, 64, 96, 300, 512, 543, 700, 1100]
    bodies = [W.ellipse(n, a=0.5, b=0.5 / (1.0 + 0.2 * k), incidence_deg=3.0 * k)
              for k, n in enumerate(panels)]
    # two steps release up to 2 M np = 6 np blobs
    ps = [params(capacity=max(4096, 8 * n), ux=1.0 + 0.1 * k, seed=k + 1)
          for k, n in enumerate(panels)]
    group = ctx.sims(ps, bodies)
    for p, (bx, bz), g in zip(ps, bodies, group):
        alone = ctx.sim(p, bx, bz)
        assert g.save() == alone.save(), g.np
        # and the two step alike
        for s in (g, alone):
            s.push_uniforms(np.random.default_rng(g.np).random(1 << 16))
            s.step(2)
            s.check()
        assert g.save() == alone.save(), g.np
        alone.close()
        g.close()


def test_group_create_is_all_or_nothing(ctx):
    """One bad body (an open contour) fails the whole group with its index in
    the message; nothing of the group stays allocated."""
    used0, _ = ctx.memory()
    good = W.circle(64)
    bad = (good[0][:-1], good[1][:-1])  # last point not the first
    with pytest.raises(Exception, match="simulation 2"):
        ctx.sims([params(capacity=4096)] * 3, [good, good, bad])
    assert ctx.memory()[0] == used0


def test_diffusion_inject_matches(ctx, port):
    bx, bz = W.circle(64)
    p = params(nu=1e-3, dt=0.01)
    s = ctx.sim(p, bx, bz)
    x, z, g, sg = _random_state(5000, 12, bx, bz)
    s.set_blobs(x, z, g, sg)
    R = port.mt_stream(42, 2 * 5000 + 100)
    s.push_uniforms(R)
    s.phase(N.PHASE_DIFFUSE)
    x0, z0 = port.diffuse(x, z, R, p.nu, p.dt)
    d = s.blobs()
    assert close(d["x"], x0, 1e-15) and close(d["z"], z0, 1e-15)


def test_diffusion_philox_statistics(ctx):
    """Counter-based walk: zero mean, variance 2 nu dt per axis (Box-Muller)."""
    bx, bz = W.circle(64)
    p = params(rng=N.RNG_PHILOX, nu=1e-3, dt=0.01, seed=99, capacity=1 << 20)
    s = ctx.sim(p, bx, bz)
    n = 1 << 20
    zeros = np.zeros(n)
    s.set_blobs(zeros + 10.0, zeros + 10.0, zeros + 1e-3, zeros + 0.1)
    s.phase(N.PHASE_DIFFUSE)
    d = s.blobs()
    dx, dz = d["x"] - 10.0, d["z"] - 10.0
    var = 2 * p.nu * p.dt
    se = np.sqrt(var / n)
    assert abs(dx.mean()) < 5 * se and abs(dz.mean()) < 5 * se
    assert abs(dx.var() / var - 1) < 0.01 and abs(dz.var() / var - 1) < 0.01
    assert abs(np.corrcoef(dx, dz)[0, 1]) < 0.01
    s.close()


@pytest.mark.parametrize("M", [1, 3, 10])
def test_release_counts_and_positions(ctx, port, M):
    bx, bz = W.circle(128)
    p = params(max_numpanelvort=M)
    s = ctx.sim(p, bx, bz)
    rng = np.random.default_rng(M)
    gam = rng.normal(0, 1, 128)
    s.set_gamma(gam)
    R = port.mt_stream(7, 5000)
    s.push_uniforms(R)
    s.phase(N.PHASE_RELEASE)
    counts, (x0, z0, c0, s0) = port.release(bx, bz, gam, M, p.nu, p.dt, p.cutoff_exp, R)
    d = s.blobs()
    assert s.n == int(counts.sum())
    assert close(d["x"], x0, 1e-14) and close(d["z"], z0, 1e-14)
    assert np.array_equal(d["circ"], c0)
    assert np.array_equal(d["sigma"], s0)
    assert np.all(d["id"] == 0)
    consumed, _ = s.rng_position()
    assert consumed == int(counts.sum())
    s.close()


def test_release_failure_status(ctx):
    """All panel circulations zero -> 0/0 counts: the reference throws
    VortexException; the device raises DVM_ERR_RELEASE and leaves state alone."""
    bx, bz = W.circle(32)
    s = ctx.sim(params(), bx, bz)
    s.set_gamma(np.zeros(32))
    s.push_uniforms(np.full(1000, 0.5))
    s.phase(N.PHASE_RELEASE)
    assert s.status() == N.ERR_RELEASE
    assert s.n == 0
    s.clear_status()
    s.close()


def _crossing_cloud(bx, bz, n, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, 0.7, n)
    th = rng.uniform(0, 2 * np.pi, n)
    x, z = r * np.cos(th), r * np.sin(th)
    x[:5] = bx[:5]  # exactly on contour vertices
    z[:5] = bz[:5]
    return x, z


@pytest.mark.parametrize("body", ["circle", "rsquare", "joukowski"])
def test_reflect_matches(ctx, port, body):
    bx, bz = {"circle": W.circle(128), "rsquare": W.rounded_square(200),
              "joukowski": W.joukowski(160, 0.12, 10.0)}[body]
    s = ctx.sim(params(surface_cross=N.REFLECT), bx, bz)
    x, z = _crossing_cloud(bx, bz, 20000, 5)
    g = np.full(x.size, 1e-3)
    s.set_blobs(x, z, g, g)
    s.phase(N.PHASE_REFLECT)
    x0, z0, moved = port.reflect(bx, bz, x, z)
    d = s.blobs()
    assert moved > 1000
    assert np.array_equal(d["x"] != x, x0 != x)  # same blobs moved
    assert close(d["x"], x0, 1e-14) and close(d["z"], z0, 1e-14)
    s.close()


@pytest.mark.parametrize("body", ["circle", "joukowski"])
def test_delete_stable_compaction(ctx, port, body):
    bx, bz = W.circle(128) if body == "circle" else W.joukowski(160, 0.12, 10.0)
    s = ctx.sim(params(surface_cross=N.DELETE, capacity=40000), bx, bz)
    x, z = _crossing_cloud(bx, bz, 30000, 6)
    g = np.arange(x.size, dtype=np.float64)
    s.set_blobs(x, z, g, g + 1)
    s.phase(N.PHASE_DELETE)
    keep = port.keep_flags(bx, bz, x, z).astype(bool)
    d = s.blobs()
    assert s.n == int(keep.sum())
    assert np.array_equal(d["circ"], g[keep])  # order preserved
    assert np.array_equal(d["x"], x[keep])
    assert np.array_equal(d["id"], np.arange(keep.sum(), dtype=np.uint32))
    s.close()


@pytest.mark.parametrize("n,frac", [(300_000, 0.01), (60_000, 0.6), (20_000, 1.0)])
def test_delete_inplace_moves_all_arrays(ctx, port, n, frac):
    """In-place compaction over many 1024-blob tiles: every one of the eight
    arrays of the kept blobs (velocities included, as delete_inside copies
    them, src/VortexSheet.cpp:424-437) in order, IDs renumbered."""
    bx, bz = W.circle(128)
    rng = np.random.default_rng(int(n * 10 + frac * 7))
    inside = rng.random(n) < frac
    r = np.where(inside, 0.45 * np.sqrt(rng.random(n)), 0.55 + 2.5 * rng.random(n))
    th = rng.uniform(0, 2 * np.pi, n)
    x, z = r * np.cos(th), r * np.sin(th)
    g = rng.normal(0, 1e-3, n)
    s = ctx.sim(params(surface_cross=N.DELETE, capacity=n, ux=1.0), bx, bz)
    s.set_blobs(x, z, g, np.full(n, 0.05))
    for ph in (N.PHASE_BIOTSAVART, N.PHASE_SOLVE, N.PHASE_SHEETBC):
        s.phase(ph)
    before = s.blobs()
    s.phase(N.PHASE_DELETE)
    s.check()
    keep = port.keep_flags(bx, bz, x, z).astype(bool)
    after = s.blobs()
    assert s.n == int(keep.sum())
    for key in ("x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"):
        assert np.array_equal(after[key], before[key][keep]), key
    assert np.array_equal(after["id"], np.arange(keep.sum(), dtype=np.uint32))
    s.close()


def test_delete_batched_equals_alone(ctx):
    """DELETE simulations stepped together (one compaction launch over all of
    them) give the same bits as each stepped alone."""
    bodies = [W.circle(96), W.joukowski(160, 0.12, 10.0), W.ellipse(128, 0.5, 0.25, 10.0)]
    clouds = []
    for k, (bx, bz) in enumerate(bodies):
        x, z = _crossing_cloud(bx, bz, 20_000 + 15_000 * k, 40 + k)
        g = np.random.default_rng(50 + k).normal(0, 1e-3, x.size)
        clouds.append((x, z, g, np.full(x.size, 0.05)))

    def make():
        out = []
        for k, (bx, bz) in enumerate(bodies):
            p = params(surface_cross=N.DELETE, rng=N.RNG_PHILOX, seed=70 + k, ux=1.0,
                       capacity=80_000, precision=N.F32 if k % 2 else N.F64)
            sim = ctx.sim(p, bx, bz)
            sim.set_blobs(*clouds[k])
            out.append(sim)
        return out

    mix = make()
    ctx.step_batch(mix, 4, use_graph=True)
    alone = make()
    for sim in alone:
        sim.step(4)
    for a, b in zip(mix, alone):
        a.check()
        b.check()
        da, db = a.blobs(), b.blobs()
        assert da["x"].size == db["x"].size
        for key in ("x", "z", "circ", "sigma", "id"):
            assert np.array_equal(da[key], db[key]), key
        a.close()
        b.close()


def test_delete_nothing_keeps_ids(ctx):
    bx, bz = W.circle(64)
    s = ctx.sim(params(surface_cross=N.DELETE), bx, bz)
    x = np.linspace(2, 3, 100)
    s.set_blobs(x, x, x, x)
    s.phase(N.PHASE_DELETE)
    assert s.n == 100 and np.array_equal(s.blobs()["x"], x)


def test_loads_match(ctx, port):
    bx, bz = W.circle(128)
    p = params()
    s = ctx.sim(p, bx, bz)
    gam = np.random.default_rng(1).normal(0, 1, 128)
    s.set_gamma(gam)
    s.phase(N.PHASE_LOADS)
    fx, fz, cd, cl = s.loads()
    fx0, fz0 = port.loads(gam, port.sheet_geometry(bx, bz), p.rho, p.dt, 3.0)
    assert abs(fx - fx0) <= 1e-12 * abs(fx0) and abs(fz - fz0) <= 1e-12 * max(abs(fz0), 1)
    assert abs(cd - fx0 / (0.5 * 1.0 * 1.0 * 9.0)) <= 1e-12 * abs(cd)


def _run_pair(ctx, port, p, bx, bz, steps, x=None, seed_blobs=None):
    """GPU (inject mode, F64) vs the oracle port on the same mt19937 stream."""
    s = ctx.sim(p, bx, bz)
    o = port.sim(oparams(p, steps), bx, bz)
    if x is not None:
        s.set_blobs(*x)
        o.set_blobs(*x)
    s.push_uniforms(port.mt_stream(p.seed, 3_000_000))
    hist = []
    for k in range(steps):
        s.step(1)
        s.check()
        o.step(1)
        d, e = s.blobs(), o.blobs()
        hist.append((k, s.n, o.n))
        assert s.n == o.n, f"step {k}: N {s.n} vs {o.n}"
        assert np.array_equal(d["id"], e["id"])
        sc = max(1.0, np.max(np.abs(e["x"])))
        assert np.max(np.abs(d["x"] - e["x"])) <= 1e-9 * sc, f"step {k}"
        assert np.max(np.abs(d["z"] - e["z"])) <= 1e-9 * sc, f"step {k}"
        assert close(s.gamma(), o.gamma(), 1e-7)
        fx, fz, _, _ = s.loads()
        fx0, fz0, _ = o.forces()
        assert abs(fx - fx0) <= 1e-7 * max(1, abs(fx0)) and abs(fz - fz0) <= 1e-7 * max(1, abs(fz0))
    return s, o, hist


def test_cylinder_reflect_euler_steps_match(ctx, port):
    """The reference's cylinder fixture flow (tests/fixtures/test_configs/
    cylinder_test.xml: REFLECT, Euler, dt 0.005, nu 1e-3, ux 3) on a 128-panel
    R=0.5 circle: 20 full steps, inject mode, FP64."""
    bx, bz = W.circle(128)
    p = params(seed=1)
    _run_pair(ctx, port, p, bx, bz, 20)


def test_rk3_delete_steps_match(ctx, port):
    bx, bz = W.circle(64)
    p = params(seed=5, scheme=N.RK3, surface_cross=N.DELETE)
    _run_pair(ctx, port, p, bx, bz, 8)


def test_step_counter_and_batch_equals_single(ctx, port):
    """Two sims stepped in one batch equal the same sims stepped alone."""
    bx, bz = W.circle(96)
    p = params(seed=3, rng=N.RNG_PHILOX, precision=N.F32)
    a = ctx.sim(p, bx, bz)
    b = ctx.sim(p, bx, bz)
    x = _random_state(4000, 3, bx, bz)
    a.set_blobs(*x)
    b.set_blobs(*x)
    ctx.step_batch([a], 3, use_graph=False)
    bx2, bz2 = W.ellipse(120, 0.5, 0.2)
    c = ctx.sim(p, bx2, bz2)
    c.set_blobs(*_random_state(2000, 4, bx2, bz2))
    ctx.step_batch([b, c], 3, use_graph=True)
    a.check(); b.check(); c.check()
    da, db = a.blobs(), b.blobs()
    assert a.n == b.n and a.step_number() == 3
    for k in ("x", "z", "circ", "u", "w", "uvs", "wvs"):
        assert np.array_equal(da[k], db[k]), k
    assert np.array_equal(a.gamma(), b.gamma())
