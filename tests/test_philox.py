"""Philox4x32-10 known-answer tests.

CPU: the numpy restatement (tests/philox_ref.py) reproduces the published
Random123 vectors.  GPU: the device generator behind DVM_RNG_PHILOX
(dvm_philox4x32_10) reproduces the same vectors and the restatement on random
counters and keys bit for bit, and one Philox diffusion step of a simulation
moves every blob by exactly the Box-Muller displacement of its own block
(counter = blob index, step, 0, stream 0; key = the seed), to the last few
ulps of the FP64 log / cos / sin.
"""
import numpy as np
import pytest

from tests.philox_ref import KAT, philox4x32_10, uniforms2


def test_restatement_matches_published_vectors():
    for ctr, key, want in KAT:
        assert tuple(int(v) for v in philox4x32_10([ctr], [key])[0]) == want


@pytest.mark.gpu
def test_device_generator_known_answers():
    from dvmpp_b200 import native as N

    ctr = np.array([c for c, _, _ in KAT], dtype=np.uint32)
    key = np.array([k for _, k, _ in KAT], dtype=np.uint32)
    want = np.array([w for _, _, w in KAT], dtype=np.uint32)
    assert np.array_equal(N.philox4x32_10(ctr, key), want)
    rng = np.random.default_rng(8)
    ctr = rng.integers(0, 2**32, (100_000, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2**32, (100_000, 2), dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(N.philox4x32_10(ctr, key), philox4x32_10(ctr, key))


@pytest.mark.gpu
def test_philox_walk_is_the_generator_plus_box_muller(ctx):
    from dvmpp_b200 import native as N
    from dvmpp_b200 import workloads as W

    seed = 0x1234_5678_9ABC
    nu, dt = 2e-3, 0.005
    bx, bz = W.circle(64)
    n = 50_000
    sim = ctx.sim(N.Params(nu=nu, dt=dt, rng=N.RNG_PHILOX, seed=seed, capacity=n), bx, bz)
    rng = np.random.default_rng(9)
    x, z = rng.uniform(1, 5, n), rng.uniform(-2, 2, n)
    sim.set_blobs(x, z, np.zeros(n), np.full(n, 0.05))
    sim.phase(N.PHASE_DIFFUSE)  # step 0
    d = sim.blobs()
    i = np.arange(n, dtype=np.uint64)
    ctr = np.stack([i, np.zeros(n, np.uint64), np.zeros(n, np.uint64), np.zeros(n, np.uint64)], 1)
    key = np.tile(np.array([seed & 0xFFFFFFFF, seed >> 32], dtype=np.uint64), (n, 1))
    r1, r2 = uniforms2(philox4x32_10(ctr, key))
    rrw = np.sqrt((4.0 * nu * dt) * np.log(1.0 / r1))
    th = 2.0 * np.pi * r2
    ex, ez = rrw * np.cos(th), rrw * np.sin(th)
    scale = np.max(rrw)
    assert np.max(np.abs((d["x"] - x) - ex)) <= 1e-13 * scale
    assert np.max(np.abs((d["z"] - z) - ez)) <= 1e-13 * scale
    sim.close()
