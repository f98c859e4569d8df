"""CPU-only checks: the C-ABI library loads and exports every symbol that
include/dvm_cuda.h declares; the oracle reproduces the reference's own
known-answer tests and the committed golden vectors (tests/golden/)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from dvmpp_b200 import native
from oracle.pyoracle import Port, SimParams, have_port

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def declared_symbols():
    text = open(native.HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(dvm_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree():
    decl = declared_symbols()
    assert len(decl) >= 30
    assert sorted(native.SIGNATURES) == decl


def test_library_exports_every_declared_symbol():
    lib = native.load()  # loads without a GPU; no compute call is made
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.dvm_abi_version() == 1
    assert lib.dvm_status_string(native.ERR_RELEASE) == b"negative PanelNewVort in release"


def test_no_device_is_reported_not_faked():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(native.DvmError) as e:
        native.Context(0)
    assert e.value.status in (native.ERR_NO_DEVICE, native.ERR_CUDA)


@pytest.fixture(scope="module")
def port():
    if not have_port():
        pytest.skip("oracle not built")
    return Port()


def test_oracle_reference_known_answers(port):
    # tests/unit/test_VelocityKernel.cpp:99-125
    d, G, s = 2.0, 1.0, 0.01
    u, w = port.direct_self([-d / 2, d / 2], [0, 0], [G, -G], [s, s])
    e = G / (2 * math.pi * d)
    assert abs(w[0] - e) <= 0.01 * e and abs(u[0]) < 1e-6
    # tests/unit/test_VelocityKernel.cpp:58-71
    u, w = port.direct_self([0.0], [0.0], [1.0], [0.1])
    assert u[0] == 0.0 and w[0] == 0.0
    # tests/unit/test_VelocityKernel.cpp:73-97
    u, w = port.direct_at([0.0], [0.0], [1.0], [0.1], [1.0], [0.0])
    assert abs(u[0]) < 1e-10 and abs(w[0] - 1 / (2 * math.pi)) < 0.01
    # tests/regression/test_CylinderFlow.cpp:26-71 (walk statistics, seed 42)
    R = port.mt_stream(42, 2000)
    x, z = port.diffuse(np.zeros(1000), np.zeros(1000), R, 1e-3, 0.01)
    spread = math.sqrt(4e-3 * 0.01)
    assert abs(x.mean()) < 0.1 and 0.5 * spread < x.std(ddof=1) < 2 * spread


def _golden(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} missing")
    return np.load(p)


def test_oracle_vs_golden_kernels(port):
    g = _golden("kernels.npz")
    u, w = port.direct_self(g["x"], g["z"], g["circ"], g["sigma"])
    assert np.array_equal(u, g["u_self"]) and np.array_equal(w, g["w_self"])
    u, w = port.direct_at(g["x"], g["z"], g["circ"], g["sigma"], g["tx"], g["tz"])
    assert np.array_equal(u, g["u_at"]) and np.array_equal(w, g["w_at"])
    assert np.array_equal(port.mt_stream(int(g["seed"]), g["stream"].size), g["stream"])


def test_oracle_vs_golden_sheet(port):
    g = _golden("sheet.npz")
    A = port.influence_matrix(g["bx"], g["bz"])
    assert np.array_equal(A, g["A"])
    geo = port.sheet_geometry(g["bx"], g["bz"])
    b = port.sheet_rhs(geo, 3.0, 0.0, g["x"], g["z"], g["circ"], g["sigma"])
    assert np.array_equal(b, g["b"])
    gam = port.sheet_solve(A, b)
    assert np.array_equal(gam, g["gamma"])
    uvs, wvs = port.sheet_on_blobs(geo, gam, g["x"], g["z"])
    assert np.array_equal(uvs, g["uvs"]) and np.array_equal(wvs, g["wvs"])


def test_oracle_vs_golden_cylinder_run(port):
    """10 steps of the reference's cylinder fixture configuration
    (tests/fixtures/test_configs/cylinder_test.xml with its 20-panel body)."""
    g = _golden("cylinder_fixture.npz")
    p = SimParams(rho=1.0, nu=1e-3, dt=0.005, ux=3.0, uz=0.0, cutoff_exp=0.675,
                  max_numpanelvort=3, scheme="euler", surface_cross="REFLECT", seed=42, steps=10)
    s = port.sim(p, g["bx"], g["bz"])
    for k in range(10):
        s.step()
        assert s.n == int(g["n"][k])
        assert np.array_equal(s.gamma(), g["gamma"][k])
        fx, fz, _ = s.forces()
        assert fx == g["fx"][k] and fz == g["fz"][k]
    b = s.blobs()
    assert np.array_equal(b["x"], g["x_final"]) and np.array_equal(b["z"], g["z_final"])
