"""State dump and resume (dvm_sim_save / dvm_sim_restore).

A simulation stepped k steps, saved, restored into a fresh context and
stepped m more gives the same bits as the uninterrupted k + m steps: every
blob array and ID, gamma, the loads, the step counter and the random
stream's position -- in inject mode (the reference's mt19937 stream, with
uniforms pushed but not consumed carried in the dump) and with the Philox
walk, for Euler / REFLECT and RK3 / DELETE, FP64 and FP32.  The reference
has no resume; its de-facto dump is the per-step text file of every blob
(src/VortexBlobs.cpp:322-325).
"""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _snapshot(sim):
    d = sim.blobs()
    d["gamma"] = sim.gamma()
    d["loads"] = np.array(sim.loads())
    d["step"] = sim.step_number()
    d["rng"] = sim.rng_position()
    return d


@pytest.mark.parametrize("rng,scheme,cross,prec", [
    (N.RNG_INJECT, N.EULER, N.REFLECT, N.F64),
    (N.RNG_PHILOX, N.RK3, N.DELETE, N.F32),
    (N.RNG_PHILOX, N.EULER, N.REFLECT, N.F32),
])
def test_save_restore_continue_is_bitwise(port, rng, scheme, cross, prec):
    bx, bz = W.joukowski(120, 0.12, 8.0) if scheme == N.RK3 else W.circle(96)
    p = N.Params(ux=1.0, nu=2e-3, rng=rng, scheme=scheme, surface_cross=cross, precision=prec,
                 seed=21, capacity=40_000, rng_capacity=400_000)
    x, z, g, s = W.wake(6000, 22, W.core_size(bx, bz))
    stream = port.mt_stream(21, 300_000)
    k, m = 3, 4

    ctx_a = N.Context(0)
    a = ctx_a.sim(p, bx, bz)
    a.set_blobs(x, z, g, s)
    if rng == N.RNG_INJECT:
        a.push_uniforms(stream)
    a.step(k + m)
    a.check()
    want = _snapshot(a)
    a.close()
    ctx_a.close()

    ctx_b = N.Context(0)
    b = ctx_b.sim(p, bx, bz)
    b.set_blobs(x, z, g, s)
    if rng == N.RNG_INJECT:
        b.push_uniforms(stream)
    b.step(k)
    b.check()
    state = b.save()
    mid = _snapshot(b)
    b.close()
    ctx_b.close()

    ctx_c = N.Context(0)  # a fresh context
    c = ctx_c.restore(state)
    got_mid = _snapshot(c)
    for key in mid:
        assert np.array_equal(np.asarray(got_mid[key]), np.asarray(mid[key])), key
    c.step(m)
    c.check()
    got = _snapshot(c)
    assert c.save() != state
    c.close()
    ctx_c.close()
    assert got["x"].size == want["x"].size
    for key in want:
        assert np.array_equal(np.asarray(got[key]), np.asarray(want[key])), key


def test_restore_rejects_foreign_or_damaged_buffers(ctx):
    bx, bz = W.circle(64)
    sim = ctx.sim(N.Params(capacity=2048), bx, bz)
    sim.set_blobs(*W.wake(100, 3, 0.08))
    state = sim.save()
    sim.close()
    for bad in (b"", b"x" * 64, state[:-8], state + b"\0" * 8,
                b"NOTSTATE" + state[8:]):
        with pytest.raises(N.DvmError) as e:
            ctx.restore(bad)
        assert e.value.status == N.ERR_ARG
