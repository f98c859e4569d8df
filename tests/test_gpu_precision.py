"""Precision of the FP32-compensated path against the all-FP64 path on the
sheet-solve workload (ellipse at 20 degrees incidence, RK3), at a size that
runs in seconds: 256 panels, a 16 k-blob wake, 4 steps.  Bounds (the
serving-path contract): velocity fields rel L2 <= 1e-5 on one identical
state, gamma rel L2 <= 1e-5, Cd within 0.5 % of the FP64 run; the QR +
refinement solve equals an independent least-squares solve to 1e-10."""
import pytest

from dvmpp_b200 import cases

pytestmark = pytest.mark.gpu


def test_fp32_path_within_bounds_of_fp64():
    r = cases.run_precision(steps=4, n_wake=1 << 14, npanels=256)
    s = r["solve"]
    assert s["qr_refined_vs_lstsq"] <= 1e-10, s
    assert s["f32_rhs_qr_refined_vs_f64"] <= 1e-5, s
    st = r["same_state"]
    for key in ("u", "w", "uvs", "wvs"):
        assert st[key + "_rel_l2"] <= 1e-5, (key, st)
    assert st["gamma_rel_l2"] <= 1e-5, st
    run = r["run"]
    assert run["steps_with_equal_n"] == 4, run
    assert run["max_gamma_rel_l2"] <= 1e-4, run
    assert run["max_cd_rel"] <= 5e-3, run
