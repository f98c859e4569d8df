"""The C++ drop-in host classes (dvmpp_b200/host) on the GPU.

1. The reference's own unit, integration and regression test sources
   (tests/*/*.cpp of gdeskos/DVMpp), compiled unmodified against the drop-in
   classes by tests/cpp/Makefile, must all pass.
2. DVMBase(xml, stamp) + solve-style stepping of the drop-in, fed the same XML
   and body file as the reference, must write the same per-step output files
   (the reference's formats: _vortex_num.dat exactly; _gamma.dat, _loads.dat,
   _vortex.dat to the 6 significant digits the reference prints)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from dvmpp_b200 import workloads as W
from oracle.pyoracle import SimParams, write_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "_build", "ref_tests_on_b200")
HOST_SO = os.path.join(ROOT, "dvmpp_b200", "lib", "libdvmpp_host.so")


def test_reference_test_suite_passes_on_dropin(tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("tests/cpp/_build/ref_tests_on_b200 not built (needs the reference tree)")
    r = subprocess.run([EXE], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    tail = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else r.stderr
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "0 failed" in tail


def _rows(path, skip):
    with open(path) as f:
        lines = f.read().splitlines()[skip:]
    return [[float(v) for v in ln.replace("\t", " ").split()] for ln in lines if ln.strip()]


@pytest.mark.parametrize("cross,scheme,steps", [("REFLECT", "euler", 10), ("DELETE", "RK3", 5)])
def test_dvmbase_dropin_writes_reference_outputs(tmp_path, ref, cross, scheme, steps):
    host = C.CDLL(HOST_SO)
    host.dvmpp_host_run_xml.argtypes = [C.c_char_p, C.c_char_p, C.c_uint, C.c_int, C.c_int,
                                        C.POINTER(C.c_ulonglong), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
    host.dvmpp_host_last_error.restype = C.c_char_p
    bx, bz = W.circle(64)
    p = SimParams(seed=42, steps=steps, surface_cross=cross, scheme=scheme)
    dref, dgpu = str(tmp_path / "ref"), str(tmp_path / "gpu")
    xml_ref = write_case(dref, p, bx, bz, stamp="case")
    xml_gpu = write_case(dgpu, p, bx, bz, stamp="case")
    rs = ref.sim(p, bx, bz, workdir=dref)
    for _ in range(steps):
        rs.step()
        rs.write_outputs()
    del rs
    n = C.c_ulonglong()
    fx, fz = C.c_double(), C.c_double()
    rc = host.dvmpp_host_run_xml(xml_gpu.encode(), b"ref", steps, 1, 1, C.byref(n), C.byref(fx),
                                 C.byref(fz))
    assert rc == 0, host.dvmpp_host_last_error()
    # blob counts per step: exact
    assert _rows(f"{dref}/ref_vortex_num.dat", 1) == _rows(f"{dgpu}/ref_vortex_num.dat", 1)
    for name, skip in (("gamma", 4), ("loads", 1), ("vortex", 4)):
        a = np.array(_rows(f"{dref}/ref_{name}.dat", skip))
        b = np.array(_rows(f"{dgpu}/ref_{name}.dat", skip))
        assert a.shape == b.shape, name
        tol = 2e-5 * np.maximum(1.0, np.abs(a)) if name != "loads" else 1e-4 * np.maximum(1.0, np.abs(a))
        assert np.all(np.abs(a - b) <= tol), (name, float(np.max(np.abs(a - b))))
