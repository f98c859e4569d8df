"""Edge cases of the whole step on the GPU (C ABI): the reference's ABSORB
branch is its REFLECT (src/DVMBase.cpp:107-118, "TODO"), so the two modes give
bitwise-equal trajectories; a release that would overflow the simulation's
capacity, and an injected uniform stream that runs short, stop that
simulation with a status code and leave its blob count unchanged (the
reference would grow its arrays or read past its stream); a failed
simulation does not disturb the others of its batch."""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _params(**kw):
    p = N.Params(capacity=kw.pop("capacity", 1 << 16), rng=N.RNG_PHILOX, seed=5,
                 rng_capacity=kw.pop("rng_capacity", 1 << 20))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _cloud(n, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.45, 0.9, n)
    th = rng.uniform(0, 2 * np.pi, n)
    g = rng.normal(0, 1e-3, n)
    return r * np.cos(th), r * np.sin(th), g - g.mean(), np.full(n, 0.08)


def test_absorb_equals_reflect(ctx):
    bx, bz = W.circle(96)
    x, z, g, s = _cloud(3000, 1)
    out = {}
    for mode in (N.ABSORB, N.REFLECT):
        sim = ctx.sim(_params(surface_cross=mode, nu=5e-3), bx, bz)
        sim.set_blobs(x, z, g, s)
        sim.step(6)
        sim.check()
        out[mode] = sim.blobs()
        sim.close()
    a, r = out[N.ABSORB], out[N.REFLECT]
    assert a["x"].size == r["x"].size
    for key in ("x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"):
        assert np.array_equal(a[key], r[key]), key


def test_capacity_overflow_stops_the_simulation_only(ctx):
    bx, bz = W.circle(128)
    small = ctx.sim(_params(capacity=1024), bx, bz)   # (M+1) * 128 = 512 blobs per step at most
    other = ctx.sim(_params(capacity=1 << 16), bx, bz)
    for _ in range(6):
        ctx.step_batch([small, other], 1, use_graph=False)
    assert small.status() == N.ERR_CAPACITY
    assert ctx.batch_status([small, other]) == [N.ERR_CAPACITY, N.OK]
    n_stop = small.n
    assert 0 < n_stop <= 1024
    ctx.step_batch([small, other], 1, use_graph=False)
    assert small.n == n_stop  # a failed simulation is frozen
    other.check()
    assert other.n > n_stop   # the healthy one kept stepping
    small.clear_status()
    small.close()
    other.close()


def test_injected_stream_exhausted(ctx):
    bx, bz = W.circle(64)
    sim = ctx.sim(_params(rng=N.RNG_INJECT, capacity=1 << 14, rng_capacity=1 << 14), bx, bz)
    x, z, g, s = _cloud(2000, 2)
    sim.set_blobs(x, z, g, s)
    sim.push_uniforms(np.full(100, 0.5))   # fewer than the 2 per blob the walk needs
    sim.step(1)
    assert sim.status() == N.ERR_RNG
    assert sim.n == 2000
    sim.clear_status()
    sim.close()


def test_create_rejects_bad_contours_and_allocates_nothing(ctx):
    bx, bz = W.circle(32)
    used0 = ctx.memory()[0]
    bad = [(bx[:-1], bz[:-1]),                                    # not closed
           (np.insert(bx, 4, bx[4]), np.insert(bz, 4, bz[4])),    # zero-length panel
           (np.where(np.arange(bx.size) == 3, np.nan, bx), bz),   # non-finite point
           (np.array([0.0, 1.0, 0.0]), np.array([0.0, 0.0, 0.0]))]  # two panels
    for xb, zb in bad:
        with pytest.raises(N.DvmError) as e:
            ctx.sim(_params(), xb, zb)
        assert e.value.status == N.ERR_ARG
    assert ctx.memory()[0] == used0


def test_set_blobs_rejects_non_finite_and_keeps_state(ctx):
    bx, bz = W.circle(64)
    sim = ctx.sim(_params(), bx, bz)
    x, z, g, s = _cloud(500, 3)
    sim.set_blobs(x, z, g, s)
    before = sim.blobs()
    for arr in range(4):
        vals = [a.copy() for a in (x, z, g, s)]
        vals[arr][123] = np.nan if arr % 2 == 0 else np.inf
        with pytest.raises(N.DvmError) as e:
            sim.set_blobs(*vals)
        assert e.value.status == N.ERR_ARG
    after = sim.blobs()
    assert sim.n == 500
    for key in ("x", "z", "circ", "sigma"):
        assert np.array_equal(before[key], after[key])
    sim.close()


def test_batch_pushes_reject_a_simulation_listed_twice(ctx):
    bx, bz = W.circle(64)
    sim = ctx.sim(_params(rng=N.RNG_INJECT, rng_capacity=1 << 12), bx, bz)
    other = ctx.sim(_params(rng=N.RNG_INJECT, rng_capacity=1 << 12), bx, bz)
    u = np.full(64, 0.5)
    for push in (ctx.batch_push_uniforms, ctx.batch_push_uniforms_async):
        with pytest.raises(N.DvmError) as e:
            push([sim, other, sim], [u, u, u], [64, 64, 64])
        assert e.value.status == N.ERR_ARG
        assert sim.rng_position() == (0, 0)  # nothing was pushed
    ctx.batch_push_uniforms([sim, other], [u, u], [64, 64])
    assert sim.rng_position() == (0, 64) and other.rng_position() == (0, 64)
    sim.close()
    other.close()
