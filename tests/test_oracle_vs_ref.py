"""The C restatement (oracle/dvm_oracle.c) against the reference's own sources
compiled unmodified (oracle/_ref/libdvmref.so): bit-for-bit equality.

Skipped where the reference build is absent (it is built from the reference
tree by oracle/Makefile and travels with the working tree)."""
import numpy as np
import pytest

from dvmpp_b200 import workloads as W
from oracle.pyoracle import SimParams


def test_direct_kernels_bitwise(port, ref):
    x, z, g, s = W.wake(2500, 31, 0.0818804)
    assert all(np.array_equal(a, b) for a, b in zip(port.direct_self(x, z, g, s),
                                                     ref.direct_self(x, z, g, s)))
    tx, tz = W.collocation_circle(100)
    tx = np.concatenate([tx, x[:5]])
    tz = np.concatenate([tz, z[:5]])
    assert all(np.array_equal(a, b) for a, b in zip(port.direct_at(x, z, g, s, tx, tz),
                                                     ref.direct_at(x, z, g, s, tx, tz)))


def test_random_stream_bitwise(port, ref):
    for seed in (0, 1, 42, 12345):
        assert np.array_equal(port.mt_stream(seed, 5000), ref.random_stream(seed, 5000))


@pytest.mark.parametrize("scheme,cross,npan,steps", [
    ("euler", "REFLECT", 128, 20),
    ("RK3", "DELETE", 64, 8),
    ("euler", "ABSORB", 40, 10),
])
def test_full_steps_bitwise(port, ref, scheme, cross, npan, steps):
    bx, bz = W.circle(npan)
    p = SimParams(scheme=scheme, surface_cross=cross, seed=7, steps=steps)
    rs, ps = ref.sim(p, bx, bz), port.sim(p, bx, bz)
    assert np.array_equal(rs.infm(), port.influence_matrix(bx, bz))
    for k in range(steps):
        rs.step()
        ps.step()
        a, b = rs.blobs(), ps.blobs()
        for key in ("x", "z", "circ", "sigma", "u", "w", "uvs", "wvs", "id"):
            assert np.array_equal(a[key], b[key]), (k, key)
        assert np.array_equal(rs.gamma(), ps.gamma())
        assert rs.forces() == ps.forces()


def test_phases_bitwise_on_a_wake(port, ref):
    """Each compute_step phase separately, from the same injected state."""
    bx, bz = W.ellipse(96, 0.5, 0.25, 20.0)
    x, z, g, s = W.wake(3000, 5, W.core_size(bx, bz))
    p = SimParams(seed=3)
    rs, ps = ref.sim(p, bx, bz), port.sim(p, bx, bz)
    rs.set_blobs(x, z, g, s)
    ps.set_blobs(x, z, g, s)
    for phase in (0, 1, 2, 4, 5, 9, 7):
        rs.phase(phase)
        ps.phase(phase)
        a, b = rs.blobs(), ps.blobs()
        for key in ("x", "z", "u", "w", "uvs", "wvs", "circ", "sigma"):
            assert np.array_equal(a[key], b[key]), (phase, key)
        assert np.array_equal(rs.gamma(), ps.gamma()), phase


def _merge_case(n, seed):
    rng = np.random.default_rng(seed)
    d = {"x": rng.uniform(0, 2, n), "z": rng.uniform(-1, 1, n),
         "circ": rng.normal(0, 1e-3, n), "sigma": rng.uniform(0.02, 0.05, n)}
    for k in ("u", "w", "uvs", "wvs"):
        d[k] = rng.normal(0, 1, n)
    d["id"] = np.arange(n, dtype=np.uint32)
    d["circ"][5] = 0.0              # zero circulation: merges at any distance
    d["circ"][6] = -d["circ"][7]    # a cancelling pair: skipped
    d["x"][9], d["z"][9] = d["x"][8], d["z"][8]  # coincident blobs
    return d


@pytest.mark.parametrize("thr", [0.0, 1e-7, 1e-6, 1e-5])
def test_merge_blobs_bitwise(port, ref, thr):
    """VortexBlobs::merge_blobs (src/VortexBlobs.cpp:110-209): the oracle's
    restatement against the reference build, all 8 arrays and the IDs."""
    d = _merge_case(3000, 3)
    a, ca = port.merge_blobs(d, thr)
    b, cb = ref.merge_blobs(d, thr)
    assert ca == cb
    for k in a:
        assert np.array_equal(a[k], b[k]), k
