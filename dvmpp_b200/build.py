"""Build the in-tree native libraries.

    python -m dvmpp_b200.build            # libdvm_cuda.so (+ host C++ library)
    python -m dvmpp_b200.build --oracle   # also the CPU oracle (oracle/_ref)

nvcc cross-compiles for sm_100a without a GPU.  Outputs land next to the
package (dvmpp_b200/lib/), so they travel with the working tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
LIB_DIR = os.path.join(HERE, "lib")
BUILD_DIR = os.path.join(HERE, "_build")
CUDA_SO = os.path.join(LIB_DIR, "libdvm_cuda.so")
HOST_SO = os.path.join(LIB_DIR, "libdvmpp_host.so")

CU_SOURCES = ["k_biot_savart.cu", "k_sheet.cu", "k_book.cu", "k_remesh.cu", "k_merge.cu",
              "dvm_capi.cu",
              "dvm_serve.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return r


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_cuda(verbose=False, force=False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "dvm_cuda.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, os.path.splitext(src)[0] + ".o")
        if force or _stale(o, [s] + headers):
            _run([nvcc, *ARCH, *NVCC_FLAGS, "-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _stale(CUDA_SO, objs):
        _run([nvcc, *ARCH, "-shared", "-o", CUDA_SO, *objs, "-lcudart_static", "-lrt", "-ldl",
              "-lpthread"], verbose)
    return CUDA_SO


def build_host(verbose=False, force=False) -> str | None:
    """C++17 drop-in classes (reference interfaces) over libdvm_cuda.so."""
    if not os.path.isdir(HOST):
        return None
    srcs = sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp"))
    if not srcs:
        return None
    hdrs = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".hpp")]
    if force or _stale(HOST_SO, srcs + hdrs + [CUDA_SO]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + HOST,
              "-I" + os.path.join(ROOT, "include"), *srcs, "-o", HOST_SO, "-L" + LIB_DIR,
              "-ldvm_cuda", "-Wl,-rpath,$ORIGIN"], verbose)
    return HOST_SO


def build_oracle(verbose=False) -> None:
    """The CPU oracle (test infrastructure): the C restatement always, and the
    reference's own sources when they are present on this machine."""
    odir = os.path.join(ROOT, "oracle")
    targets = ["oracle"]
    ref = reference_dir()
    ref_present = ref is not None
    extra = [f"REF={ref}"] if ref_present else []
    if ref_present:
        targets.append("ref")
    _run(["make", "-s", "-C", odir, *targets, *extra], verbose)
    if ref_present:  # the reference's own C++ tests against the drop-in classes
        _run(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp"), *extra], verbose)


def reference_dir() -> str | None:
    """The reference source tree (gdeskos/DVMpp): $DVM_REFERENCE, else a
    checkout named `reference` beside this repository; None when neither
    holds a src/ directory (the oracle is then the C restatement alone)."""
    cand = os.environ.get("DVM_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
    return cand if os.path.isdir(os.path.join(cand, "src")) else None


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build_cuda(a.verbose, a.force))
    h = build_host(a.verbose, a.force)
    if h:
        print(h)
    if a.oracle:
        build_oracle(a.verbose)


if __name__ == "__main__":
    main()
