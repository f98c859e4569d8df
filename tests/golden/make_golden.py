"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own sources compiled by oracle/Makefile
(oracle/_ref/libdvmref.so) -- only where the reference tree exists:

    make -C oracle ref && python tests/golden/make_golden.py

The body of the sheet and cylinder cases is the reference's own fixture
tests/fixtures/test_data/simple_body.txt (20 panels, R = 0.5), run with the
parameters of tests/fixtures/test_configs/cylinder_test.xml.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyoracle import Ref, SimParams  # noqa: E402

REFERENCE = os.environ.get("DVM_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def main():
    ref = Ref()
    rng = np.random.default_rng(2024)
    # kernels: 400 blobs in a 2x2 box, 64 targets
    n = 400
    x, z = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    circ, sigma = rng.normal(0, 1e-2, n), np.full(n, 0.0818804)
    tx, tz = rng.uniform(-1.2, 1.2, 64), rng.uniform(-1.2, 1.2, 64)
    us, ws = ref.direct_self(x, z, circ, sigma)
    ua, wa = ref.direct_at(x, z, circ, sigma, tx, tz)
    stream = ref.random_stream(42, 600)
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), x=x, z=z, circ=circ, sigma=sigma,
                        tx=tx, tz=tz, u_self=us, w_self=ws, u_at=ua, w_at=wa, seed=42,
                        stream=stream)

    body = np.loadtxt(os.path.join(REFERENCE, "tests/fixtures/test_data/simple_body.txt"))
    bx, bz = body[:, 0].copy(), body[:, 1].copy()
    p = SimParams(rho=1.0, nu=1e-3, dt=0.005, ux=3.0, uz=0.0, cutoff_exp=0.675,
                  max_numpanelvort=3, scheme="euler", surface_cross="REFLECT", seed=42, steps=10)
    # sheet: influence matrix, rhs, gamma, sheet-on-blob for 300 blobs around the body
    s = ref.sim(p, bx, bz)
    A = s.infm()
    r = 0.5 + rng.uniform(0.01, 1.0, 300)
    th = rng.uniform(0, 2 * np.pi, 300)
    bxs, bzs = r * np.cos(th), r * np.sin(th)
    bc, bs = rng.normal(0, 1e-2, 300), np.full(300, 0.2)
    s.set_blobs(bxs, bzs, bc, bs)
    s.phase(1)  # solvevortexsheet
    gamma = s.gamma()
    s.phase(2)  # vortexsheetbc
    d = s.blobs()
    # right-hand side recomputed from the reference's own velocities at the collocation points
    sh = s.sheet()
    uc, wc = ref.direct_at(bxs, bzs, bc, bs, sh["xc"], sh["zc"])
    np.savez_compressed(os.path.join(HERE, "sheet.npz"), bx=bx, bz=bz, A=A, x=bxs, z=bzs,
                        circ=bc, sigma=bs, gamma=gamma, uvs=d["uvs"], wvs=d["wvs"],
                        b=_rhs(sh, bxs, bzs, bc, bs, 3.0, 0.0))
    # the cylinder fixture run
    s = ref.sim(p, bx, bz)
    ns, gs, fxs, fzs = [], [], [], []
    for _ in range(10):
        s.step()
        ns.append(s.n)
        gs.append(s.gamma())
        fx, fz, _ = s.forces()
        fxs.append(fx)
        fzs.append(fz)
    b = s.blobs()
    np.savez_compressed(os.path.join(HERE, "cylinder_fixture.npz"), bx=bx, bz=bz,
                        n=np.array(ns), gamma=np.array(gs), fx=np.array(fxs), fz=np.array(fzs),
                        x_final=b["x"], z_final=b["z"])
    print("golden vectors written to", HERE)


def _rhs(sh, x, z, circ, sigma, Ux, Uz):
    """b exactly as src/VortexSheet.cpp:181-210 forms it (same loop order)."""
    npan = sh["xc"].size
    b = np.empty(npan + 1)
    rpi2 = 1.0 / (2.0 * 3.14159265358979323846)
    for i in range(npan):
        u = w = 0.0
        for j in range(x.size):
            dx = sh["xc"][i] - x[j]
            dz = sh["zc"][i] - z[j]
            r2 = dx * dx + dz * dz
            thr = 10 * sigma[j] ** 2
            rs = 1.0 / sigma[j] ** 2
            K = (1.0 - np.exp(-r2 * rs)) / r2 if r2 < thr else 1.0 / r2
            u -= K * dz * circ[j]
            w += K * dx * circ[j]
        u *= rpi2
        w *= rpi2
        b[i] = (Ux + u) * sh["enx"][i] + (Uz + w) * sh["enz"][i]
    tc = 0.0
    for c in circ:
        tc += c
    b[npan] = -tc
    return b


if __name__ == "__main__":
    main()
