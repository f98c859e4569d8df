"""dvm_biot_savart_at_noalloc: the velocity-at-targets entry point that
allocates nothing, for callers that cannot call cudaMalloc (their device
memory belongs to a host framework's allocator or pool, or an allocation's
implicit synchronisation is not acceptable where they run).

Checked through the C ABI against the existing entry point
(dvm_biot_savart_at_device) on two calls in a row, within the tolerances the
other Biot-Savart tests use.  The caller's buffers come from torch here; the
entry point itself only launches kernels on its fixed in-library scratch.
This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12   # relative to the field's max, as in test_gpu_biot_savart.py
F32_REL_L2 = 1e-5


def _dev(torch, a):
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_no_alloc_matches_existing_entry_point_two_calls():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    lib = N.load()
    ctx = N.Context(0)
    try:
        cases = [(6000, 300, N.F32, 1), (30000, 256, N.F64, 0)]
        for call, (ns, nt, prec, skip) in enumerate(cases):
            x, z, g, s = W.wake(ns, 70 + call, 0.0818804)
            tx, tz = W.collocation_circle(nt, 0.5 + 0.1 * call)
            tx[:3], tz[:3] = x[:3], z[:3]  # targets on sources exercise the close-pair rule
            d = [_dev(torch, a) for a in (x, z, g, s, tx, tz)]
            u1 = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
            w1 = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
            u2, w2 = torch.empty_like(u1), torch.empty_like(w1)
            torch.cuda.synchronize()
            rc = lib.dvm_biot_savart_at_noalloc(*[_ptr(t) for t in d[:4]], ns, _ptr(d[4]),
                                                _ptr(d[5]), nt, _ptr(u1), _ptr(w1), prec, skip,
                                                None)
            assert rc == N.OK, lib.dvm_last_error()
            torch.cuda.synchronize()
            rc = lib.dvm_biot_savart_at_device(ctx.h, *[_ptr(t) for t in d[:4]], ns, _ptr(d[4]),
                                               _ptr(d[5]), nt, _ptr(u2), _ptr(w2), prec, skip)
            assert rc == N.OK, lib.dvm_last_error()
            ctx.sync()
            a_u, a_w = u1.cpu().numpy(), w1.cpu().numpy()
            b_u, b_w = u2.cpu().numpy(), w2.cpu().numpy()
            # Without the close-pair skip a target on a source divides 0/0 (NaN),
            # as the reference's solvevortexsheet loop does; both entry points must
            # agree on where, and every other entry must be written.
            nan_a, nan_b = np.isnan(a_u) | np.isnan(a_w), np.isnan(b_u) | np.isnan(b_w)
            assert np.array_equal(nan_a, nan_b)
            assert nan_a[:3].all() if not skip else not nan_a.any()
            assert not nan_a[3:].any()
            a_u, a_w, b_u, b_w = a_u[3:], a_w[3:], b_u[3:], b_w[3:]
            if prec == N.F64:
                sc = max(np.max(np.abs(b_u)), np.max(np.abs(b_w)))
                assert np.max(np.abs(a_u - b_u)) <= F64_TOL * sc
                assert np.max(np.abs(a_w - b_w)) <= F64_TOL * sc
            else:
                assert np.linalg.norm(a_u - b_u) <= F32_REL_L2 * np.linalg.norm(b_u)
                assert np.linalg.norm(a_w - b_w) <= F32_REL_L2 * np.linalg.norm(b_w)
    finally:
        ctx.close()


def test_no_alloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    lib = N.load()
    one = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = _ptr(one)
    # 2^22 sources x 256 targets needs 1024 chunks x 256 partials: one chunk more
    # than the fixed array holds beside the job record
    rc = lib.dvm_biot_savart_at_noalloc(p, p, p, p, 1 << 22, p, p, 256, p, p, N.F32, 1, None)
    assert rc == N.ERR_ARG
    assert b"262080" in lib.dvm_last_error()
    # few sources but 262 144 padded targets: also one row of partials too many
    rc = lib.dvm_biot_savart_at_noalloc(p, p, p, p, 100, p, p, 262_080, p, p, N.F32, 1, None)
    assert rc == N.ERR_ARG


def _compare(lib, ctx, torch, x, z, g, s, tx, tz, prec, skip):
    ns, nt = x.size, tx.size
    d = [_dev(torch, a) for a in (x, z, g, s, tx, tz)]
    u1 = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
    w1 = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
    u2, w2 = torch.empty_like(u1), torch.empty_like(w1)
    torch.cuda.synchronize()
    rc = lib.dvm_biot_savart_at_noalloc(*[_ptr(t) for t in d[:4]], ns, _ptr(d[4]), _ptr(d[5]), nt,
                                        _ptr(u1), _ptr(w1), prec, skip, None)
    assert rc == N.OK, lib.dvm_last_error()
    torch.cuda.synchronize()
    rc = lib.dvm_biot_savart_at_device(ctx.h, *[_ptr(t) for t in d[:4]], ns, _ptr(d[4]),
                                       _ptr(d[5]), nt, _ptr(u2), _ptr(w2), prec, skip)
    assert rc == N.OK, lib.dvm_last_error()
    ctx.sync()
    a_u, a_w = u1.cpu().numpy(), w1.cpu().numpy()
    b_u, b_w = u2.cpu().numpy(), w2.cpu().numpy()
    assert np.isfinite(a_u).all() and np.isfinite(a_w).all()
    assert np.linalg.norm(a_u - b_u) <= F32_REL_L2 * np.linalg.norm(b_u)
    assert np.linalg.norm(a_w - b_w) <= F32_REL_L2 * np.linalg.norm(b_w)


def test_no_alloc_at_its_size_limit_and_with_many_targets():
    """The largest accepted call (1023 source chunks x 256 targets: the partials
    fill the array up to the job record in its tail) and a call with fewer
    sources than one chunk but 100 000 targets, each against the existing
    entry point."""
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    lib = N.load()
    ctx = N.Context(0)
    try:
        x, z, g, s = W.wake(4096 * 1023, 91, 0.0818804)
        tx, tz = W.collocation_circle(256, 0.55)
        _compare(lib, ctx, torch, x, z, g, s, tx, tz, N.F32, 1)
        x, z, g, s = W.wake(3000, 92, 0.0818804)
        rng = np.random.default_rng(93)
        tx, tz = rng.uniform(-2, 20, 100_000), rng.normal(0, 1, 100_000)
        _compare(lib, ctx, torch, x, z, g, s, tx, tz, N.F32, 1)
    finally:
        ctx.close()
