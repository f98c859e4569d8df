"""Coefficients of the polynomial evaluations in the FP32 kernels: the
sheet-on-blob kernel (k_sheet.cu, sheet_pair_f32) and the blob-on-blob core
kernel (k_biot_savart.cu, core_kernel): fitted here, pasted there.

    python dvmpp_b200/csrc/fit_polys.py

Method: Lawson's algorithm (C. L. Lawson, 1961) -- iteratively reweighted
least squares on a dense Chebyshev grid, which converges to the minimax
(equi-oscillating) approximation -- applied to the relative error:

  L(x) ~ log1p(x) / x        on x in [-1/4, 1/4],  degree 7 in x
  T(s) ~ atan(t) / t, s = t^2 on t in [0, 1/4],    degree 3 in s (small angles)
  G(s) ~ atan(t) / t, s = t^2 on t in [0, 1],      degree 9 in s (any angle,
                                                   after |t| = min / max)
  P(t) ~ (1 - exp(-t)) / t  on t in [0, 1/2],       degree 5 in t (the
                                                   regularised core below
                                                   t = r^2 / sigma^2 = 1/2)

Each fit prints its coefficients (constant term first) and the maximum
relative error of the FP32 Horner evaluation (numpy float32, fused
multiply-adds emulated in float64 then rounded) over a dense grid, against
the float64 function.
"""
import numpy as np


def lawson(f, a, b, deg, var=lambda x: x, iters=200, npts=4000):
    """Minimax-relative polynomial in var(x) approximating f on [a, b]."""
    k = np.arange(npts)
    x = 0.5 * (a + b) + 0.5 * (b - a) * np.cos(np.pi * (k + 0.5) / npts)
    y = f(x)
    V = np.vander(var(x), deg + 1, increasing=True) / y[:, None]  # relative error rows
    w = np.full(npts, 1.0 / npts)
    c = None
    for _ in range(iters):
        sw = np.sqrt(w)
        c, *_ = np.linalg.lstsq(V * sw[:, None], sw, rcond=None)
        e = np.abs(V @ c - 1.0)
        w = w * e
        w /= w.sum()
    return c


def horner_f32(c, v):
    v = v.astype(np.float32)
    p = np.full_like(v, np.float32(c[-1]))
    for ck in c[-2::-1]:
        p = (p.astype(np.float64) * v.astype(np.float64) + np.float32(ck)).astype(np.float32)
    return p


def fitted(name, src, c, f, xs, var, post):
    """The fit rounded to FP32 and its maximum relative error in FP32 Horner form."""
    c32 = [np.float32(v) for v in c]
    got = post(xs.astype(np.float32), horner_f32(c32, var(xs)))
    ref = f(xs)
    err = float(np.max(np.abs(got.astype(np.float64) - ref) / np.abs(ref)))
    return {"name": name, "source": src, "coefficients": c32, "max_rel_err": err}


def literal(v) -> str:
    """A coefficient as the kernels spell it."""
    return f"{float(v):.9e}f"


def fits():
    """Every polynomial: name, the kernel source it is pasted into, its FP32
    coefficients (constant term first) and the error of its FP32 evaluation."""
    out = []
    # log1p(x) = x * L(x), |x| <= 1/4
    f = lambda x: np.where(x == 0, 1.0, np.log1p(x) / np.where(x == 0, 1.0, x))
    c = lawson(f, -0.25, 0.25, 7)
    xs = np.linspace(-0.25, 0.25, 200001)
    xs = xs[xs != 0]
    out.append(fitted("L (log1p, |x| <= 1/4)", "k_sheet.cu", c, lambda x: np.log1p(x), xs,
                      lambda x: x,
                      lambda x, p: (x.astype(np.float64) * p.astype(np.float64)).astype(np.float32)))

    # atan(t) = t * T(t^2), |t| <= 1/4
    g = lambda t: np.where(t == 0, 1.0, np.arctan(t) / np.where(t == 0, 1.0, t))
    c = lawson(lambda s: g(np.sqrt(s)), 0.0, 0.0625, 3)
    ts = np.linspace(1e-6, 0.25, 200001)
    out.append(fitted("T (atan, |t| <= 1/4)", "k_sheet.cu", c, np.arctan, ts,
                      lambda t: t.astype(np.float64) ** 2,
                      lambda t, p: (t.astype(np.float64) * p.astype(np.float64)).astype(np.float32)))

    # atan(t) = t * G(t^2), 0 <= t <= 1
    c = lawson(lambda s: g(np.sqrt(s)), 0.0, 1.0, 9)
    ts = np.linspace(1e-6, 1.0, 400001)
    out.append(fitted("G (atan, |t| <= 1)", "k_sheet.cu", c, np.arctan, ts,
                      lambda t: t.astype(np.float64) ** 2,
                      lambda t, p: (t.astype(np.float64) * p.astype(np.float64)).astype(np.float32)))

    # (1 - exp(-t)) / t on 0 <= t <= 1/2 (the value at t = 0 is 1)
    h = lambda t: np.where(t == 0, 1.0, -np.expm1(-t) / np.where(t == 0, 1.0, t))
    c = lawson(h, 0.0, 0.5, 5)
    ts = np.linspace(0.0, 0.5, 200001)
    out.append(fitted("P (core, t <= 1/2)", "k_biot_savart.cu", c, h, ts, lambda t: t,
                      lambda t, p: p))
    return out


def main():
    for r in fits():
        print(f"{r['name']} ({r['source']}): max rel err (FP32 Horner) {r['max_rel_err']:.3e}")
        print("  " + ", ".join(literal(v) for v in r["coefficients"]))


if __name__ == "__main__":
    main()
