"""Input validation without a GPU.

* The drop-in host classes (dvmpp_b200/host): malformed XML raises
  dvm::XMLParseException, comments / CDATA / entities parse, a body file that
  is not a closed contour of finite points with >= 3 non-degenerate panels
  raises dvm::FileIOException (tests/cpu_cpp/input_validation_check.cpp).
* The C ABI: dvm_sim_create checks the contour and the parameters before it
  looks at the context, so the same rejections are visible here through
  ctypes (DVM_ERR_ARG and the reason in dvm_last_error), and
  dvm_sim_set_blobs rejects a null simulation.
"""
import ctypes as C
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from dvmpp_b200 import native as N
from dvmpp_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "dvmpp_b200", "host")
LIB = os.path.join(ROOT, "dvmpp_b200", "lib")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_host_classes_reject_bad_xml_and_bodies(tmp_path):
    if not os.path.exists(os.path.join(LIB, "libdvmpp_host.so")):
        pytest.skip("libdvmpp_host.so not built")
    exe = str(tmp_path / "check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + HOST, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpu_cpp", "input_validation_check.cpp"), "-o", exe,
                    "-L" + LIB, "-ldvmpp_host", "-ldvm_cuda", "-Wl,-rpath," + LIB], check=True,
                   capture_output=True, text=True)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


def _create(bx, bz, params=None):
    lib = N.load()
    p = (params or N.Params()).c()
    bx, bz = np.ascontiguousarray(bx, float), np.ascontiguousarray(bz, float)
    h = C.c_void_p()
    rc = lib.dvm_sim_create(None, C.byref(p), bx.ctypes.data_as(C.POINTER(C.c_double)),
                            bz.ctypes.data_as(C.POINTER(C.c_double)), bx.size, C.byref(h))
    return rc, lib.dvm_last_error().decode()


@pytest.mark.parametrize("case,fragment", [
    ("open", "not closed"),
    ("repeated", "zero length"),
    ("nan", "not finite"),
    ("inf", "not finite"),
    ("two_panels", "at least 3 panels"),
    ("point", "at least 3 panels"),
    ("collapsed", "all the same"),
])
def test_abi_rejects_bad_contours(case, fragment):
    bx, bz = W.circle(32)
    if case == "open":
        bx, bz = bx[:-1], bz[:-1]
    elif case == "repeated":
        bx, bz = np.insert(bx, 5, bx[5]), np.insert(bz, 5, bz[5])
    elif case == "nan":
        bx = bx.copy()
        bx[7] = math.nan
    elif case == "inf":
        bz = bz.copy()
        bz[0] = bz[-1] = math.inf
    elif case == "two_panels":
        bx, bz = np.array([0.0, 1.0, 0.0]), np.array([0.0, 0.0, 0.0])
    elif case == "point":
        bx, bz = np.array([0.0]), np.array([0.0])
    elif case == "collapsed":
        bx, bz = np.zeros(6), np.zeros(6)
    rc, msg = _create(bx, bz)
    assert rc == N.ERR_ARG and fragment in msg, (rc, msg)


def test_abi_rejects_non_finite_parameters():
    bx, bz = W.circle(32)
    for field in ("ux", "uz", "cutoff_exp", "dt", "nu", "rho"):
        p = N.Params()
        setattr(p, field, math.nan)
        rc, msg = _create(bx, bz, p)
        assert rc == N.ERR_ARG, (field, rc, msg)


def test_abi_valid_contour_reaches_the_context_check():
    # a good body passes validation and fails only on the missing context
    bx, bz = W.ellipse(64, 0.5, 0.25, 10.0)
    rc, msg = _create(bx, bz)
    assert rc == N.ERR_ARG and "ctx is null" in msg, (rc, msg)


def test_abi_null_simulation_arguments():
    lib = N.load()
    x = np.zeros(4)
    p = x.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.dvm_sim_set_blobs(None, 4, p, p, p, p) == N.ERR_ARG
    assert lib.dvm_sim_push_uniforms(None, p, 4) == N.ERR_ARG
    assert lib.dvm_sim_rng_position(None, None, None) == N.ERR_ARG
