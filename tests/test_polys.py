"""CPU checks of the FP32 kernels' own polynomial evaluations.

dvmpp_b200/csrc/fit_polys.py fits them (Lawson's algorithm, minimax relative
error) and the kernels carry the fitted FP32 coefficients as literals.  This
re-runs the fits and requires (1) every non-constant coefficient to appear,
spelled the same, in the kernel source it belongs to, (2) every constant term
to be exactly 1 (the kernels write it as 1), and (3) the FP32 Horner error to
stay within the bound the kernels' comments state: 1.8e-7 relative for the
sheet-on-blob log / atan evaluations, 6.5e-8 (the degree-8 Taylor series it
replaced) for the blob-on-blob core kernel.
"""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dvmpp_b200", "csrc")

BOUNDS = {"k_sheet.cu": 1.8e-7, "k_biot_savart.cu": 6.5e-8}


def _fits():
    spec = importlib.util.spec_from_file_location("fit_polys", os.path.join(CSRC, "fit_polys.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod, mod.fits()


MOD, FITS = _fits()


@pytest.mark.parametrize("fit", FITS, ids=[f["name"].split()[0] for f in FITS])
def test_kernel_coefficients_are_the_fit(fit):
    with open(os.path.join(CSRC, fit["source"])) as f:
        src = f.read()
    c = fit["coefficients"]
    assert c[0] == np.float32(1.0), fit["name"]
    for v in c[1:]:
        assert MOD.literal(v) in src, (fit["name"], MOD.literal(v))
    assert fit["max_rel_err"] <= BOUNDS[fit["source"]], (fit["name"], fit["max_rel_err"])
