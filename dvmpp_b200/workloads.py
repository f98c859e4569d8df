"""Seeded synthetic bodies and wakes (no dataset is involved anywhere).

Bodies are closed, counter-clockwise contours with the first point repeated
last -- the reference's domain_file format (src/VortexSheet.cpp:56-76,
outward normals for CCW order at :93-96).
"""
from __future__ import annotations

import math

import numpy as np


def _close(x, z):
    x = np.append(x, x[0])
    z = np.append(z, z[0])
    return x, z


def _ccw(x, z):
    area = 0.5 * np.sum(x[:-1] * np.roll(z[:-1], -1) - np.roll(x[:-1], -1) * z[:-1])
    if area < 0:
        x, z = x[::-1].copy(), z[::-1].copy()
    return x, z


def circle(npanels: int, radius: float = 0.5):
    """Circle starting at (R, 0), CCW; npanels + 1 points."""
    t = 2.0 * np.pi * np.arange(npanels) / npanels
    return _close(radius * np.cos(t), radius * np.sin(t))


def ellipse(npanels: int, a: float = 0.5, b: float = 0.25, incidence_deg: float = 0.0):
    """Ellipse with semi-axes a, b, rotated nose-up by the incidence angle."""
    t = 2.0 * np.pi * np.arange(npanels) / npanels
    x, z = a * np.cos(t), b * np.sin(t)
    al = -math.radians(incidence_deg)
    xr = x * math.cos(al) - z * math.sin(al)
    zr = x * math.sin(al) + z * math.cos(al)
    return _close(*_ccw(xr, zr))


def rounded_square(npanels: int, side: float = 1.0, radius: float = 0.05):
    """Square of the given side with rounded corners, sampled by arc length."""
    h = side / 2.0 - radius
    straight = 2.0 * h
    arc = 0.5 * math.pi * radius
    per = 4.0 * (straight + arc)
    s = per * np.arange(npanels) / npanels
    xs, zs = np.empty(npanels), np.empty(npanels)
    # segments: right edge (up), top-right arc, top edge (left), ... CCW from (side/2, -h)
    for k, sv in enumerate(s):
        q = sv
        for side_i in range(4):
            if q < straight:
                pos = -h + q
                pts = [(h + radius, pos), (-pos, h + radius), (-h - radius, -pos), (pos, -h - radius)]
                xs[k], zs[k] = pts[side_i]
                break
            q -= straight
            if q < arc:
                ang = q / radius + side_i * 0.5 * math.pi
                cx = [h, -h, -h, h][side_i]
                cz = [h, h, -h, -h][side_i]
                xs[k], zs[k] = cx + radius * math.cos(ang), cz + radius * math.sin(ang)
                break
            q -= arc
    return _close(*_ccw(xs, zs))


def joukowski(npanels: int, thickness: float = 0.12, aoa_deg: float = 0.0, chord: float = 1.0):
    """Symmetric Joukowski airfoil (circle through the critical point z=1,
    centre (-eps, 0), mapped by zeta + 1/zeta), scaled to the chord and
    rotated nose-up by the angle of attack."""
    eps = thickness / 1.299
    a = 1.0 + eps
    t = 2.0 * np.pi * np.arange(npanels) / npanels
    zeta = -eps + a * np.exp(1j * t)
    w = zeta + 1.0 / zeta
    x, z = w.real, w.imag
    x = (x - x.min()) / (x.max() - x.min()) * chord - 0.5 * chord
    z = z / (w.real.max() - w.real.min()) * chord
    al = -math.radians(aoa_deg)
    xr = x * math.cos(al) - z * math.sin(al)
    zr = x * math.sin(al) + z * math.cos(al)
    return _close(*_ccw(xr, zr))


def body_radius(x, z) -> float:
    return float(np.max(np.hypot(x, z)))


def core_size(x, z, cutoff_exp: float = 0.675) -> float:
    """sigma = ds^q of the body's mean panel (src/VortexSheet.cpp:325)."""
    ds = np.hypot(np.diff(x), np.diff(z))
    return float(np.mean(ds) ** cutoff_exp)


def wake(n: int, seed: int, sigma: float, scale: float = 1.0):
    """Blob set of the standalone N-body workload: 70 % in a wake with
    x ~ U[0.5, 20], z ~ N(0, 1); 30 % uniform in the annulus 0.5 < r < 1.5
    (r = sqrt(U[0.25, 2.25])); Gamma ~ N(0, 1e-3) shifted so the FP64 sum is
    zero (the residual goes on the last blob).  Lengths scale with `scale`."""
    rng = np.random.default_rng(seed)
    nw = int(round(0.7 * n))
    na = n - nw
    x = np.empty(n)
    z = np.empty(n)
    x[:nw] = rng.uniform(0.5, 20.0, nw)
    z[:nw] = rng.normal(0.0, 1.0, nw)
    r = np.sqrt(rng.uniform(0.25, 2.25, na))
    th = rng.uniform(0.0, 2.0 * np.pi, na)
    x[nw:] = r * np.cos(th)
    z[nw:] = r * np.sin(th)
    perm = rng.permutation(n)
    x, z = x[perm] * scale, z[perm] * scale
    g = rng.normal(0.0, 1e-3, n)
    g -= g.mean()
    g[-1] -= math.fsum(g)
    s = np.full(n, sigma)
    return x, z, g, s


def collocation_circle(n: int = 256, radius: float = 0.5):
    t = 2.0 * np.pi * (np.arange(n) + 0.5) / n
    return radius * np.cos(t), radius * np.sin(t)


def batched_instances(count: int = 64, seed: int = 4):
    """Mixed bodies of the batched workload: circle R=0.5, ellipses of aspect
    U[1,4], rounded squares (side 1, corner radius 0.05); panels log-uniform in
    [64, 512]; wakes log-uniform in [1e4, 4e5] blobs, distributed as `wake`
    scaled to the body radius."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        kind = ("circle", "ellipse", "rsquare")[int(rng.integers(0, 3))]
        npan = int(round(math.exp(rng.uniform(math.log(64), math.log(512)))))
        nb = int(round(math.exp(rng.uniform(math.log(1e4), math.log(4e5)))))
        if kind == "circle":
            bx, bz = circle(npan)
        elif kind == "ellipse":
            asp = float(rng.uniform(1.0, 4.0))
            bx, bz = ellipse(npan, 0.5, 0.5 / asp)
        else:
            bx, bz = rounded_square(npan)
        R = body_radius(bx, bz)
        sig = core_size(bx, bz)
        x, z, g, s = wake(nb, seed * 1000 + k, sig, scale=R / 0.5)
        out.append(dict(kind=kind, npanels=npan, nblobs=nb, body=(bx, bz), blobs=(x, z, g, s)))
    return out


def serving_requests(count: int = 1000, seed: int = 7, rate_per_s: float = 20.0,
                     steps_range=(100, 2000), panels_range=(64, 512)):
    """Requests of the serving workload: Poisson arrivals at `rate_per_s`;
    bodies from {circle R=0.5, ellipse aspect U[1,4], rounded square,
    Joukowski thickness U[0.08,0.16] at AoA U[0,15] deg}; panels U{64..512};
    nu log-uniform [1e-4, 1e-2]; ux U[1,3]; steps U{100..2000}; dt 0.005;
    REFLECT; each simulation starts with no blobs."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += rng.exponential(1.0 / rate_per_s)
        kind = ("circle", "ellipse", "rsquare", "joukowski")[int(rng.integers(0, 4))]
        npan = int(rng.integers(panels_range[0], panels_range[1] + 1))
        if kind == "circle":
            bx, bz = circle(npan)
        elif kind == "ellipse":
            bx, bz = ellipse(npan, 0.5, 0.5 / float(rng.uniform(1.0, 4.0)))
        elif kind == "rsquare":
            bx, bz = rounded_square(npan)
        else:
            bx, bz = joukowski(npan, float(rng.uniform(0.08, 0.16)), float(rng.uniform(0.0, 15.0)))
        nu = float(math.exp(rng.uniform(math.log(1e-4), math.log(1e-2))))
        ux = float(rng.uniform(1.0, 3.0))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        out.append(dict(kind=kind, npanels=npan, body=(bx, bz), nu=nu, ux=ux, steps=steps,
                        arrival=t, seed=int(rng.integers(0, 2**31 - 1))))
    return out
