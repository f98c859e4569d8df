"""Probe velocities (dvm_sim_probe) against the oracle.  The reference's
VortexSheet::probe_velocities (src/VortexSheet.cpp:559-646) is never called by
its loop and has slips (blob 0 and panel 0 skipped, only the last panel's
term kept, a sign flipped), so parity is against its intended formula, built
from oracle pieces that are pinned to the reference: the at-target blob sum
(computeInducedAt, src/VelocityKernel.cpp:69-109) + the sheet-on-point sum
(vortexsheetbc's panel formula, src/VortexSheet.cpp:217-273) + the free
stream.  FP64: 1e-12 of the field scale; FP32 instances: 1e-5."""
import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _points(x, z, n, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.52, 3.0, n)
    th = rng.uniform(0, 2 * np.pi, n)
    px, pz = r * np.cos(th), r * np.sin(th)
    px[0], pz[0] = x[7], z[7]  # a probe exactly on a blob: that pair is skipped
    return px, pz


@pytest.mark.parametrize("prec", [N.F64, N.F32])
def test_probe_matches_intended_formula(ctx, port, prec):
    bx, bz = W.ellipse(96, 0.5, 0.3, 10.0)
    p = N.Params(capacity=1 << 14, precision=prec, ux=1.5, uz=0.2)
    s = ctx.sim(p, bx, bz)
    x, z, g, sg = W.wake(4000, 21, W.core_size(bx, bz))
    s.set_blobs(x, z, g, sg)
    s.phase(N.PHASE_SOLVE)
    gamma = s.gamma()
    px, pz = _points(x, z, 300, 5)
    u, w, uvs, wvs = s.probe(px, pz)
    ub, wb = port.direct_at(x, z, g, sg, px, pz)
    us0, ws0 = port.sheet_on_blobs(port.sheet_geometry(bx, bz), gamma, px, pz)
    u0, w0 = ub + us0 + p.ux, wb + ws0 + p.uz
    tol = 1e-12 if prec == N.F64 else 1e-5
    scale = max(np.max(np.abs(u0)), np.max(np.abs(w0)))
    assert np.max(np.abs(uvs - us0)) <= 1e-12 * scale
    assert np.max(np.abs(wvs - ws0)) <= 1e-12 * scale
    assert np.max(np.abs(u - u0)) <= tol * scale
    assert np.max(np.abs(w - w0)) <= tol * scale
    # no blobs: sheet + free stream only
    s.set_blobs([], [], [], [])
    u, w, _, _ = s.probe(px, pz)
    assert np.max(np.abs(u - (us0 + p.ux))) <= 1e-12 * scale
    s.close()
