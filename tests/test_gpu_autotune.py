"""The pair-kernel autotuner: every launch shape in its search space gives
bitwise-identical steps (CTAs per SM and item order never change a target's
operation sequence, and the mutual far tiles' fixed-point sums do not depend on
the order their terms arrive in; source chunking, which would change results,
is fixed by capacity), and autotune() keeps the fastest shape for the batch's
class; shapes outside the search space are refused."""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _batch(ctx, sizes, seed=3):
    sims = []
    for k, n in enumerate(sizes):
        bx, bz = W.circle(64 + 32 * k)
        p = N.Params(capacity=n + 8192, precision=N.F32, rng=N.RNG_PHILOX, seed=seed + k,
                     ux=1.0, surface_cross=N.REFLECT)
        s = ctx.sim(p, bx, bz)
        x, z, g, sg = W.wake(n, seed + k, W.core_size(bx, bz))
        s.set_blobs(x, z, g, sg)
        sims.append(s)
    return sims


SIZES = [3000, 17000, 700, 40000, 9000]


def _run(ctx, steps=2):
    sims = _batch(ctx, SIZES)
    ctx.step_batch(sims, steps, use_graph=True)
    out = []
    for s in sims:
        s.check()
        out.append(s.blobs())
        s.close()
    return out


def test_every_shape_gives_identical_steps(ctx):
    ref = _run(ctx)
    for cand in N.tune_candidates():
        ctx.set_pair_config(-1, cand["tile"], cand["ctas_per_sm"], cand["order"])
        got = _run(ctx)
        for a, b in zip(got, ref):
            for key in ("x", "z", "u", "w", "uvs", "wvs"):
                assert np.array_equal(a[key], b[key]), (cand, key)
    ctx.set_pair_config(-1, 256, 4, 0)


def test_autotune_keeps_the_fastest_for_the_class(ctx):
    sims = _batch(ctx, SIZES)
    r = ctx.autotune(sims, reps=2)
    assert len(r["candidates"]) == len(N.tune_candidates())
    assert r["best_ms"] == min(c["ms"] for c in r["candidates"])
    assert r["best_ms"] <= r["default_ms"]
    assert r["shape_class"] == ctx.shape_class(sims)
    assert ctx.pair_config(r["shape_class"]) == r["best"]
    ctx.step_batch(sims, 2, use_graph=True)
    tuned = [s.blobs() for s in sims]
    for s in sims:
        s.check()
        s.close()
    ctx.set_pair_config(-1, 256, 4, 0)  # back to the default shape, table cleared
    ref = _run(ctx)
    for a, b in zip(tuned, ref):
        assert np.array_equal(a["u"], b["u"]) and np.array_equal(a["x"], b["x"])


def test_tuning_table_round_trip(ctx, tmp_path):
    ctx.set_pair_config(7, 256, 2, 1)
    ctx.set_pair_config(41, 256, 1, 0)
    table = ctx.tuning_table()
    assert table[7] == {"tile": 256, "ctas_per_sm": 2, "order": 1}
    assert table[41] == {"tile": 256, "ctas_per_sm": 1, "order": 0}
    path = tmp_path / "tuning.json"
    ctx.save_tuning(str(path))
    other = N.Context(0)
    other.load_tuning(str(path))
    assert other.tuning_table() == table
    other.close()
    with pytest.raises(N.DvmError):
        ctx.set_pair_config(3, 256, 5, 0)  # 1..4 CTAs per SM
    with pytest.raises(N.DvmError):
        ctx.set_pair_config(3, 128, 2, 0)  # work items are one 256-blob tile
    ctx.set_pair_config(-1, 256, 4, 0)
    assert ctx.tuning_table() == {}
