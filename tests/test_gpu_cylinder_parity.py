"""The plain-DVM cylinder configuration run to the end (150 steps, ~50 k blobs)
on the GPU in FP64 inject mode, checked against the CPU oracle at every step
(tests/parity_cylinder.py holds the run).  Blob counts must be equal at every
step; velocities, sheet strengths and loads agree to round-off, which the
chaotic flow may amplify over the run -- hence the per-quantity bounds:
  u, w, uvs, wvs, positions: rel L2 <= 1e-8
  gamma:                     rel L2 <= 1e-8
  Cd:                        rel <= 1e-6;  Cl: abs <= 1e-6"""
import pytest

from tests.parity_cylinder import run, summary
from dvmpp_b200 import native as N

pytestmark = pytest.mark.gpu


def test_cylinder_150_steps_fp64_matches_oracle(ctx, port):
    rows = run(150, N.F64, ctx=ctx, port=port)
    s = summary(rows)
    assert s["steps_with_equal_n"] == 150, s
    assert s["final_n"] > 30000
    for key in ("u", "w", "uvs", "wvs", "x"):
        assert s["max_rel_l2_" + key] <= 1e-8, (key, s)
    assert s["max_rel_l2_gamma"] <= 1e-8, s
    assert s["max_cd_rel"] <= 1e-6 and s["max_cl_abs"] <= 1e-6, s
