"""Biot-Savart parity on the GPU, through the C ABI (include/dvm_cuda.h).

Oracle: the C restatement of src/VelocityKernel.cpp:30-109 (oracle/dvm_oracle.c).
Tolerances:
  * DVM_F64: |u - u_oracle| <= 1e-12 * max|u_oracle| (the reference's per-pair
    operations; the sums run over Morton-sorted tiles and source chunks, so they
    re-associate, and exp() may differ by an ulp).
  * DVM_F32: relative L2 error <= 1e-5 (the bar for the FP32 compensated path),
    max-norm error reported.
Cases follow the reference's own tests (tests/unit/test_VelocityKernel.cpp,
tests/integration/test_BiotSavart.cpp) plus seeded random sets.
"""
import math

import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
F32_REL_L2 = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_f32_sums_scale_exactly_with_circulation(ctx):
    """The FP32 path sums velocities in 64-bit fixed point with a per-simulation
    shift from max|Gamma| and min sigma.  Scaling every Gamma by 2^k scales each
    FP32 term by 2^k exactly and moves the shift by k, so the velocities scale by
    2^k bit for bit: the fixed-point range follows the data at any magnitude."""
    x, z, g, s = W.wake(40000, 5, 0.08188)
    u0, w0 = ctx.biot_savart_self(x, z, g, s, N.F32)
    assert np.all(np.isfinite(u0)) and np.any(u0 != 0.0)
    for k in (-40, 40, 80):
        u, w = ctx.biot_savart_self(x, z, g * 2.0 ** k, s, N.F32)
        assert np.array_equal(u, u0 * 2.0 ** k) and np.array_equal(w, w0 * 2.0 ** k), k


def test_empty_and_single(ctx):
    # test_VelocityKernel.cpp:47-71
    u, w = ctx.biot_savart_self([], [], [], [], N.F64)
    assert u.size == 0 and w.size == 0
    for prec in (N.F64, N.F32):
        u, w = ctx.biot_savart_self([0.0], [0.0], [1.0], [0.1], prec)
        assert u[0] == 0.0 and w[0] == 0.0


@pytest.mark.parametrize("prec", [N.F64, N.F32])
def test_vortex_pair_analytic(ctx, prec):
    # test_VelocityKernel.cpp:99-125 and test_BiotSavart.cpp:15-51
    d, G, s = 2.0, 1.0, 0.01
    u, w = ctx.biot_savart_self([-d / 2, d / 2], [0, 0], [G, -G], [s, s], prec)
    expected = G / (2 * math.pi * d)
    assert abs(w[0] - expected) <= 0.01 * expected
    assert abs(w[1] - expected) <= 0.01 * expected
    assert abs(u[0]) < 1e-10 and abs(u[1]) < 1e-10


@pytest.mark.parametrize("prec", [N.F64, N.F32])
def test_corotating_and_leapfrog(ctx, prec):
    d, G, s = 2.0, 1.0, 0.01
    u, w = ctx.biot_savart_self([-d / 2, d / 2], [0, 0], [G, G], [s, s], prec)
    e = G / (2 * math.pi * d)
    assert abs(w[0] + e) <= 0.01 * e and abs(w[1] - e) <= 0.01 * e
    # test_BiotSavart.cpp:117-161
    x = [-1.0, -1.0, 1.0, 1.0]
    z = [0.5, -0.5, 0.5, -0.5]
    c = [1.0, -1.0, 1.0, -1.0]
    u, w = ctx.biot_savart_self(x, z, c, [0.05] * 4, prec)
    tol = 1e-10 if prec == N.F64 else 1e-6
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(w))
    assert abs(u[0] - u[2]) < tol and abs(u[1] - u[3]) < tol


def test_close_pair_finite(ctx):
    # test_BiotSavart.cpp:89-114
    for prec in (N.F64, N.F32):
        u, w = ctx.biot_savart_self([-0.0005, 0.0005], [0, 0], [1, -1], [0.1, 0.1], prec)
        assert np.all(np.isfinite(u)) and np.all(np.isfinite(w))


@pytest.mark.parametrize("n", [1, 2, 3, 255, 256, 257, 1023, 1024, 1025, 5000])
def test_self_f64_vs_oracle(ctx, port, n):
    x, z, g, s = W.wake(n, 10 + n, 0.0818804)
    u0, w0 = port.direct_self(x, z, g, s)
    u, w = ctx.biot_savart_self(x, z, g, s, N.F64)
    scale = max(np.max(np.abs(u0)), np.max(np.abs(w0)), 1e-300)
    assert np.max(np.abs(u - u0)) <= F64_TOL * scale
    assert np.max(np.abs(w - w0)) <= F64_TOL * scale


@pytest.mark.parametrize("n", [2, 100, 1024, 4097, 20000])
def test_self_f32_vs_oracle(ctx, port, n):
    x, z, g, s = W.wake(n, 20 + n, 0.0818804)
    u0, w0 = port.direct_self(x, z, g, s)
    u, w = ctx.biot_savart_self(x, z, g, s, N.F32)
    assert rel_l2(u, u0) <= F32_REL_L2, rel_l2(u, u0)
    assert rel_l2(w, w0) <= F32_REL_L2, rel_l2(w, w0)


def test_f32_edge_magnitudes(ctx, port):
    """Range edges of the fixed-point sums: no circulation anywhere gives exact
    zeros (the shift clamps); zero core sizes (every pair on the 1/r^2 branch,
    as the reference's test r2 < 10 sigma^2 then never holds) and mixed core
    sizes over three decades match the oracle (sigma = 0 used to round every
    sum to zero: the bound's minimum distance is now floored at the coordinates'
    scale).

    Without a core the velocity of a blob is dominated by its nearest
    neighbours (here down to 3.9e-4 apart), and the FP32 path's offsets are
    FP32 values relative to a 256-blob tile's first blob, so a close pair's
    dx carries ulp(tile extent) / r relative error.  A CPU emulation of that
    arithmetic gives rel-L2 4.1e-5 (sigma = 0) and 1.1e-5 (cores down to
    9e-4) against 1.1e-6 for the regular wake; exact FP64 differences would
    give 6e-8 in all three.  Those two cases are held to 1e-4."""
    x, z, g, s = W.wake(5000, 31, 0.0818804)
    u, w = ctx.biot_savart_self(x, z, np.zeros_like(g), s, N.F32)
    assert np.all(u == 0.0) and np.all(w == 0.0)
    for sig in (np.zeros_like(s), np.exp(np.random.default_rng(4).uniform(-7.0, -0.5, s.size))):
        u0, w0 = port.direct_self(x, z, g, sig)
        u, w = ctx.biot_savart_self(x, z, g, sig, N.F32)
        assert np.all(np.isfinite(u)) and np.all(np.isfinite(w))
        assert rel_l2(u, u0) <= 1e-4 and rel_l2(w, w0) <= 1e-4, (rel_l2(u, u0), rel_l2(w, w0))


def test_self_f32_clustered_boundary_layer(ctx, port):
    """Dense nascent-blob layer next to a body: close pairs dominate."""
    rng = np.random.default_rng(3)
    n = 8000
    th = rng.uniform(0, 2 * np.pi, n)
    r = 0.5 + np.abs(rng.normal(0, 0.01, n))
    x, z = r * np.cos(th) + 3.0, r * np.sin(th) - 1.0
    g = rng.normal(0, 1e-3, n)
    s = np.full(n, 0.0818804)
    u0, w0 = port.direct_self(x, z, g, s)
    u, w = ctx.biot_savart_self(x, z, g, s, N.F32)
    assert rel_l2(u, u0) <= F32_REL_L2 and rel_l2(w, w0) <= F32_REL_L2


def test_f32_blobs_closer_than_fp32_resolution(ctx, port):
    """Nascent blobs of one panel can land closer than FP32 resolves; the FP64
    reference is finite there (K -> 1/sigma^2), so the FP32 path must be too."""
    x, z, g, s = W.wake(3000, 9, 0.0818804)
    x = np.concatenate([x, x[:50] + 1e-10, x[50:60] + 3e-8])
    z = np.concatenate([z, z[:50], z[50:60] - 2e-8])
    g = np.concatenate([g, g[:60]])
    s = np.full(x.size, 0.0818804)
    u0, w0 = port.direct_self(x, z, g, s)
    assert np.all(np.isfinite(u0))
    u, w = ctx.biot_savart_self(x, z, g, s, N.F32)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(w))
    assert rel_l2(u, u0) <= F32_REL_L2 and rel_l2(w, w0) <= F32_REL_L2


def test_coincident_distinct_blobs_match_reference_nan(ctx, port):
    """Two distinct blobs at the same point: the reference divides 0/0 (NaN)."""
    x, z = [0.0, 0.0, 1.0], [0.0, 0.0, 0.0]
    u0, w0 = port.direct_self(x, z, [1.0, 1.0, 1.0], [0.1] * 3)
    u, w = ctx.biot_savart_self(x, z, [1.0, 1.0, 1.0], [0.1] * 3, N.F64)
    assert np.array_equal(np.isnan(u), np.isnan(u0))


@pytest.mark.parametrize("prec", [N.F64, N.F32])
def test_at_targets_vs_oracle(ctx, port, prec):
    x, z, g, s = W.wake(6000, 5, 0.0818804)
    tx, tz = W.collocation_circle(256)
    tx = np.concatenate([tx, x[:10]])  # targets on blobs: r2 <= 1e-15 skipped (:89)
    tz = np.concatenate([tz, z[:10]])
    u0, w0 = port.direct_at(x, z, g, s, tx, tz)
    u, w = ctx.biot_savart_at(x, z, g, s, tx, tz, prec)
    if prec == N.F64:
        sc = np.max(np.abs(u0)) + np.max(np.abs(w0))
        assert np.max(np.abs(u - u0)) <= F64_TOL * sc and np.max(np.abs(w - w0)) <= F64_TOL * sc
    else:
        assert rel_l2(u, u0) <= F32_REL_L2 and rel_l2(w, w0) <= F32_REL_L2


def test_at_single_target_known_answer(ctx):
    # test_VelocityKernel.cpp:73-97
    for prec in (N.F64, N.F32):
        u, w = ctx.biot_savart_at([0.0], [0.0], [1.0], [0.1], [1.0], [0.0], prec)
        assert abs(u[0]) < 1e-10
        assert abs(w[0] - 1.0 / (2 * math.pi)) < 0.01


def test_large_f32_properties(ctx):
    """At 2^18 blobs (too big for the oracle here): antisymmetry of the pair
    interaction gives sum_i Gamma_i u_i ~ 0 and w = 0 for a mirrored set."""
    x, z, g, s = W.wake(1 << 18, 7, 0.0818804)
    u, w = ctx.biot_savart_self(x, z, g, s, N.F32)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(w))
    # momentum-like invariant: sum Gamma_i * u_i is zero analytically
    mom = abs(np.dot(g, u)) / (np.linalg.norm(g) * np.linalg.norm(u))
    assert mom < 1e-5
    # determinism: identical inputs give bit-identical outputs
    u2, w2 = ctx.biot_savart_self(x, z, g, s, N.F32)
    assert np.array_equal(u, u2) and np.array_equal(w, w2)
