"""Serving loop (dvm_server_*): continuous batching with HBM-budget admission.

The key property: every request's result is the same alone and in the mix.
Each simulation's random walk is keyed by its own seed (Philox counters carry
no batch position) and its pair sums are associated by its own capacity, so
the final blob state must be bit-identical between a batched run and the
serial (one request at a time) run of the same requests."""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _params(r, steps):
    M = 3
    return N.Params(nu=r["nu"], ux=r["ux"], dt=0.005, max_numpanelvort=M, rng=N.RNG_PHILOX,
                    precision=N.F32, seed=r["seed"], surface_cross=N.REFLECT,
                    capacity=steps * (M + 1) * r["npanels"] * 2 + 1024)


def _run(ctx, reqs, serial, budget=0, max_active=64):
    srv = N.Server(ctx, budget_bytes=budget, max_active=max_active, keep_state=True)
    ids = [srv.submit(_params(r, r["steps"]), *r["body"], r["steps"], r["arrival"]) for r in reqs]
    srv.run(serial=serial, realtime=False)
    out = {i: (srv.result(i), srv.final_blobs(i)) for i in ids}
    st = srv.stats()
    srv.close()
    return out, st


def test_alone_equals_in_mix(ctx):
    reqs = W.serving_requests(12, seed=11, steps_range=(5, 30), panels_range=(64, 200))
    mixed, st_m = _run(ctx, reqs, serial=False)
    alone, st_a = _run(ctx, reqs, serial=True)
    assert st_m["completed"] == len(reqs) and st_a["completed"] == len(reqs)
    assert st_m["peak_active"] > 1 and st_a["peak_active"] == 1
    for i in mixed:
        (ra, (xa, za, ca)), (rb, (xb, zb, cb)) = mixed[i], alone[i]
        assert ra["status"] == 0 and rb["status"] == 0
        assert ra["steps_done"] == reqs[i]["steps"]
        assert ra["blobs"] == rb["blobs"] and xa.size == ra["blobs"]
        assert np.array_equal(xa, xb) and np.array_equal(za, zb) and np.array_equal(ca, cb)
        assert ra["cd"] == rb["cd"] and ra["cl"] == rb["cl"]


def test_admission_respects_hbm_budget(ctx):
    reqs = W.serving_requests(10, seed=12, steps_range=(5, 15), panels_range=(64, 128))
    sizes = [N.sim_bytes(_params(r, r["steps"]), r["npanels"]) for r in reqs]
    budget = int(2.5 * max(sizes))  # at most two or three resident at once
    _, st = _run(ctx, reqs, serial=False, budget=budget)
    assert st["completed"] == len(reqs)
    assert st["peak_bytes"] <= budget
    assert 1 <= st["peak_active"] <= 3


def test_batch_state_and_uniform_calls_match_single(ctx):
    """dvm_batch_push_uniforms / dvm_batch_get_state against the per-simulation
    calls: same trajectories, same counts, positions and loads."""
    rng = np.random.default_rng(8)
    bodies = [W.circle(64), W.ellipse(96, 0.5, 0.25, 5.0), W.circle(128)]

    def make():
        out = []
        for k, (bx, bz) in enumerate(bodies):
            s = ctx.sim(N.Params(capacity=1 << 15, rng_capacity=1 << 18, seed=k), bx, bz)
            x, z, g, sg = W.wake(2000 + 500 * k, k, W.core_size(bx, bz))
            s.set_blobs(x, z, g, sg)
            out.append(s)
        return out

    a, b = make(), make()
    for step in range(3):
        us = [1.0 - rng.random(2 * s.n + 8 * s.np + 64) for s in a]
        for s, u in zip(a, us):
            s.push_uniforms(u)
        ctx.batch_push_uniforms(b, us, [u.size for u in us])
        ctx.step_batch(a, 1)
        ctx.step_batch(b, 1)
        xs = [np.empty(1 << 15) for _ in b]
        zs = [np.empty(1 << 15) for _ in b]
        cs = [np.empty(1 << 15) for _ in b]
        counts, loads = ctx.batch_get_state(b, xs, zs, cs)
        for i, s in enumerate(a):
            d = s.blobs()
            assert counts[i] == s.n
            assert np.array_equal(xs[i][:counts[i]], d["x"])
            assert np.array_equal(cs[i][:counts[i]], d["circ"])
            assert np.allclose(loads[i], s.loads(), rtol=0, atol=0)
    for s in a + b:
        s.check()
        s.close()


def test_pipelined_async_calls_match_synchronous(ctx):
    """dvm_batch_push_uniforms_async / dvm_batch_get_state_async /
    dvm_batch_wait_state in a pipelined loop (the next step's uniforms pushed
    and the next step enqueued before the previous step's state is read back)
    give the same counts, positions, circulations and loads, bit for bit, as
    the synchronous batch calls on identical simulations."""
    import torch

    rng = np.random.default_rng(9)
    bodies = [W.circle(64), W.ellipse(96, 0.5, 0.25, 5.0), W.circle(128)]
    cap, steps = 1 << 15, 4

    def make():
        out = []
        for k, (bx, bz) in enumerate(bodies):
            s = ctx.sim(N.Params(capacity=cap, rng_capacity=1 << 19, seed=k), bx, bz)
            x, z, g, sg = W.wake(2000 + 500 * k, k, W.core_size(bx, bz))
            s.set_blobs(x, z, g, sg)
            out.append(s)
        return out

    def pinned(n):
        return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()

    a, b = make(), make()
    us = [[1.0 - rng.random(2 * cap + 8 * s.np + 64) for s in a] for _ in range(steps)]
    ref = []
    for k in range(steps):  # synchronous
        ctx.batch_push_uniforms(a, us[k], [u.size for u in us[k]])
        ctx.step_batch(a, 1)
        xs, zs, cs = ([np.empty(cap) for _ in a] for _ in range(3))
        counts, loads = ctx.batch_get_state(a, xs, zs, cs)
        ref.append((counts, [x[:n].copy() for x, n in zip(xs, counts)],
                    [z[:n].copy() for z, n in zip(zs, counts)],
                    [c[:n].copy() for c, n in zip(cs, counts)], loads.copy()))
    hb = [[pinned(u.size) for u in row] for row in us]
    for row, dst in zip(us, hb):
        for u, h in zip(row, dst):
            h[:] = u
    outs = [[pinned(cap) for _ in b] for _ in range(3)]
    ctx.batch_push_uniforms_async(b, hb[0], [u.size for u in hb[0]])
    ctx.step_batch(b, 1)
    ctx.batch_get_state_async(b)
    for k in range(steps):  # pipelined
        if k + 1 < steps:
            ctx.batch_push_uniforms_async(b, hb[k + 1], [u.size for u in hb[k + 1]])
            ctx.step_batch(b, 1)
        counts, loads = ctx.batch_wait_state(*outs)
        if k + 1 < steps:
            ctx.batch_get_state_async(b)
        rc, rx, rz, rcirc, rl = ref[k]
        assert counts == rc, k
        for i in range(len(b)):
            assert np.array_equal(outs[0][i][:counts[i]], rx[i]), (k, i)
            assert np.array_equal(outs[1][i][:counts[i]], rz[i]), (k, i)
            assert np.array_equal(outs[2][i][:counts[i]], rcirc[i]), (k, i)
        assert np.array_equal(loads, rl), k
    for s in a + b:
        s.check()
        s.close()


def test_live_submissions_while_running(ctx):
    """Requests submitted from another host thread while dvm_server_run works
    (DVM_SERVE_LIVE) are admitted into the running batch, stamped at their
    submission, and give the same bits as the same requests run alone."""
    import threading
    import time

    reqs = W.serving_requests(10, seed=13, steps_range=(20, 60), panels_range=(64, 160))
    for r in reqs[:3]:
        r["steps"] = 150  # the early requests are still running when the live ones come
    srv = N.Server(ctx, max_active=64, keep_state=True)
    srv.set_option(N.SERVE_LIVE, 1)
    early = [srv.submit(_params(r, r["steps"]), *r["body"], r["steps"]) for r in reqs[:3]]
    errors = []
    run = threading.Thread(target=lambda: _guard(errors, srv.run, serial=False, realtime=True))
    run.start()
    live = []
    try:
        for r in reqs[3:]:
            time.sleep(0.05)
            live.append(srv.submit(_params(r, r["steps"]), *r["body"], r["steps"]))
        time.sleep(0.05)
        srv.close_intake()
        with pytest.raises(N.DvmError) as e:  # the intake is closed
            srv.submit(_params(reqs[0], 5), *reqs[0]["body"], 5)
        assert e.value.status == N.ERR_STATE
    finally:
        srv.close_intake()
        run.join(timeout=300)
    assert not run.is_alive() and not errors, errors
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    results = {i: (srv.result(i), srv.final_blobs(i)) for i in early + live}
    srv.close()
    # live requests were submitted after the run started: stamped then, and
    # some of them ran beside the early ones
    starts = [results[i][0]["arrival_s"] for i in live]
    assert all(a > 0 for a in starts) and starts == sorted(starts)
    assert any(results[i][0]["admitted_s"] < results[early[0]][0]["finished_s"] for i in live)
    alone, _ = _run(ctx, reqs, serial=True)
    for k, i in enumerate(early + live):
        (ra, (xa, za, ca)), (rb, (xb, zb, cb)) = results[i], alone[k]
        assert ra["status"] == 0 and ra["steps_done"] == reqs[k]["steps"]
        assert ra["blobs"] == rb["blobs"]
        assert np.array_equal(xa, xb) and np.array_equal(za, zb) and np.array_equal(ca, cb)
        assert ra["cd"] == rb["cd"] and ra["cl"] == rb["cl"]


def _guard(errors, fn, **kw):
    try:
        fn(**kw)
    except Exception as e:  # surfaced by the test thread
        errors.append(e)


def test_submit_after_run_is_refused(ctx):
    reqs = W.serving_requests(2, seed=14, steps_range=(3, 5), panels_range=(64, 80))
    srv = N.Server(ctx, max_active=4)
    for r in reqs:
        srv.submit(_params(r, r["steps"]), *r["body"], r["steps"])
    srv.run()
    with pytest.raises(N.DvmError) as e:
        srv.submit(_params(reqs[0], 3), *reqs[0]["body"], 3)
    assert e.value.status == N.ERR_STATE
    srv.close()
