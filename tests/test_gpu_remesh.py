"""Remeshing (dvm_sim_remesh / dvm_remesh) against the oracle's restatement of
the reference's BackgroundMesh (whose source is absent from the reference; its
behaviour is pinned by tests/unit/test_BackgroundMesh.cpp: M4', M6 and
truncated Gaussian tensor-product kernels, partition of unity, circulation
conservation).  M4' and M6 are bit-identical to the oracle (same summation
order, one rounding per operation); the Gaussian uses the platform exp, so it
agrees to 1e-13.  Also: circulation and (M4') first moments conserved, blobs
outside the mesh kept unchanged, the device-resident and host-array entry
points agree, capacity overflow leaves the simulation unchanged."""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _params(kernel, thr=1e-9, dx=0.02):
    return N.RemeshParams(xmin=-1.0, xmax=4.0, zmin=-1.5, zmax=1.5, dx=dx, dz=dx * 1.25,
                          sigma=0.03, circ_threshold=thr, kernel=kernel)


def _blobs(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.5, 3.5, n)
    z = np.clip(rng.normal(0.0, 0.4, n), -1.2, 1.2)  # support inside the mesh
    x[:50] = rng.uniform(-3.0, -1.05, 50)  # outside the mesh: kept as they are
    z[50:80] = rng.uniform(1.49, 1.6, 30)  # support crosses the top edge: kept
    g = rng.normal(0.0, 1e-3, n)
    return x, z, g, np.full(n, 0.05)


def _oracle(port, x, z, g, s, p):
    nx, nz = N.remesh_grid(p)
    return port.remesh(x, z, g, s, p.xmin, p.zmin, p.dx, p.dz, nx, nz, p.kernel, p.sigma,
                       p.circ_threshold)


@pytest.mark.parametrize("kernel", [N.REMESH_M4PRIME, N.REMESH_M6, N.REMESH_GAUSSIAN])
def test_remesh_matches_oracle(ctx, port, kernel):
    x, z, g, s = _blobs(20000, 3)
    p = _params(kernel, thr=1e-9 if kernel != N.REMESH_GAUSSIAN else 0.0)
    got = ctx.remesh(x, z, g, s, p)
    ref = _oracle(port, x, z, g, s, p)
    assert got[0].size == ref[0].size
    for a, b in zip(got, ref):
        if kernel == N.REMESH_GAUSSIAN:
            assert np.max(np.abs(a - b)) <= 1e-13 * max(np.max(np.abs(b)), 1e-300)
        else:
            assert np.array_equal(a, b)
    # the 80 edge / outside blobs come last, unchanged, in their order
    assert np.array_equal(got[0][-80:], x[:80]) and np.array_equal(got[2][-80:], g[:80])


@pytest.mark.parametrize("kernel", [N.REMESH_M4PRIME, N.REMESH_M6, N.REMESH_GAUSSIAN])
def test_remesh_conserves_circulation(ctx, kernel):
    x, z, g, s = _blobs(5000, 4)
    ox, oz, oc, _ = ctx.remesh(x, z, g, s, _params(kernel, thr=0.0))
    scale = np.sum(np.abs(g))
    assert abs(np.sum(oc) - np.sum(g)) <= 1e-13 * scale
    if kernel == N.REMESH_M4PRIME:  # M4' also keeps the first moments
        assert abs(np.sum(oc * ox) - np.sum(g * x)) <= 1e-12 * np.sum(np.abs(g * x))
        assert abs(np.sum(oc * oz) - np.sum(g * z)) <= 1e-12 * np.sum(np.abs(g * z))


def test_sim_remesh_in_place_equals_host_path(ctx):
    bx, bz = W.circle(64)
    x, z, g, s = _blobs(8000, 5)
    p = _params(N.REMESH_M4PRIME)
    ref = ctx.remesh(x, z, g, s, p)
    sim = ctx.sim(N.Params(capacity=200000), bx, bz)
    sim.set_blobs(x, z, g, s)
    n = sim.remesh(p)
    d = sim.blobs()
    assert n == ref[0].size == d["x"].size
    for k, key in enumerate(("x", "z", "circ", "sigma")):
        assert np.array_equal(d[key], ref[k]), key
    assert np.array_equal(d["id"], np.arange(n, dtype=np.uint32))
    assert not np.any(d["u"]) and not np.any(d["uvs"])
    # deterministic: a second remesh of the same input gives the same bits
    sim.set_blobs(x, z, g, s)
    sim.remesh(p)
    assert np.array_equal(sim.blobs()["circ"], ref[2])
    sim.close()


def test_sim_remesh_capacity_overflow_leaves_state(ctx):
    bx, bz = W.circle(64)
    x, z, g, s = _blobs(3000, 6)
    sim = ctx.sim(N.Params(capacity=4096), bx, bz)  # far fewer than the mesh's nodes
    sim.set_blobs(x, z, g, s)
    with pytest.raises(N.DvmError) as e:
        sim.remesh(_params(N.REMESH_M4PRIME, thr=0.0))
    assert e.value.status == N.ERR_CAPACITY
    sim.clear_status()
    d = sim.blobs()
    assert np.array_equal(d["x"], x) and np.array_equal(d["circ"], g)
    sim.close()


def test_steps_with_remesh_match_oracle(ctx, port):
    """Whole steps with a remesh between convection and diffusion (the
    reference's order, src/DVMBase.cpp:86-92) every third step, inject mode
    (the reference's mt19937 stream on both sides), FP64: equal blob counts,
    positions within 1e-9, sheet strengths within 1e-7."""
    from oracle.pyoracle import SimParams

    bx, bz = W.circle(64)
    p = N.Params(capacity=1 << 16, rng_capacity=1 << 22, seed=2, ux=1.0)
    op = SimParams(rho=p.rho, nu=p.nu, dt=p.dt, ux=p.ux, uz=p.uz, cutoff_exp=p.cutoff_exp,
                   max_numpanelvort=p.max_numpanelvort, scheme="euler",
                   surface_cross="REFLECT", seed=p.seed, steps=6)
    rp = N.RemeshParams(xmin=-2.0, xmax=3.0, zmin=-2.0, zmax=2.0, dx=0.05, dz=0.05, sigma=0.06,
                        circ_threshold=0.0, kernel=N.REMESH_M4PRIME)
    nx, nz = N.remesh_grid(rp)
    rng = np.random.default_rng(9)
    r = rng.uniform(0.55, 1.5, 2000)
    th = rng.uniform(0, 2 * np.pi, 2000)
    g = rng.normal(0, 1e-3, 2000)
    x0 = (r * np.cos(th), r * np.sin(th), g, np.full(2000, 0.06))
    s = ctx.sim(p, bx, bz)
    o = port.sim(op, bx, bz)
    s.set_blobs(*x0)
    o.set_blobs(*x0)
    s.push_uniforms(port.mt_stream(p.seed, 2_000_000))
    for k in range(6):
        if k % 3 != 2:
            s.step(1)
            o.step(1)
        else:
            for ph in (N.PHASE_INCREMENT, N.PHASE_CONVECT):
                s.phase(ph)
                o.phase(ph)
            s.remesh(rp)
            d = o.blobs()
            o.set_blobs(*port.remesh(d["x"], d["z"], d["circ"], d["sigma"], rp.xmin, rp.zmin,
                                     rp.dx, rp.dz, nx, nz, rp.kernel, rp.sigma,
                                     rp.circ_threshold))
            for ph in (N.PHASE_DIFFUSE, N.PHASE_RELEASE, N.PHASE_CROSS, N.PHASE_LOADS):
                s.phase(ph)
                o.phase(ph)
        s.check()
        d, e = s.blobs(), o.blobs()
        assert s.n == o.n, (k, s.n, o.n)
        sc = max(1.0, np.max(np.abs(e["x"])))
        assert np.max(np.abs(d["x"] - e["x"])) <= 1e-9 * sc, k
        assert np.max(np.abs(d["z"] - e["z"])) <= 1e-9 * sc, k
        assert np.max(np.abs(d["circ"] - e["circ"])) <= 1e-12 * np.max(np.abs(e["circ"])), k
        g0 = o.gamma()
        assert np.max(np.abs(s.gamma() - g0)) <= 1e-7 * max(np.max(np.abs(g0)), 1e-300), k
    s.close()
