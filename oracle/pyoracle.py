"""ctypes front-end to the two CPU oracles (see ``oracle/__init__.py``).

TEST INFRASTRUCTURE ONLY.  Every function mirrors one reference routine; the
C side cites the exact reference lines (gdeskos/DVMpp, ``src/...``).
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PORT_SO = os.path.join(REF_DIR, "libdvmoracle.so")
REF_SO = os.path.join(REF_DIR, "libdvmref.so")

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_up = C.POINTER(C.c_uint)


def _ptr(a):
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_u8p)
    if a.dtype == np.uint32:
        return a.ctypes.data_as(_up)
    raise TypeError(a.dtype)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class SimParams:
    """The XML parameters the hot path reads (src/XmlHandler.cpp:162-202)."""

    rho: float = 1.0
    nu: float = 1e-3
    dt: float = 0.005
    ux: float = 3.0
    uz: float = 0.0
    cutoff_exp: float = 0.675
    max_numpanelvort: int = 3
    scheme: str = "euler"          # "euler" | "RK3"
    surface_cross: str = "REFLECT"  # "DELETE" | "ABSORB" | "REFLECT"
    seed: int = 1
    steps: int = 150

    def scheme_id(self) -> int:
        return 0 if self.scheme == "euler" else 1

    def cross_id(self) -> int:
        return {"DELETE": 0, "ABSORB": 1, "REFLECT": 2}[self.surface_cross]


# --------------------------------------------------------------------------
# C port
# --------------------------------------------------------------------------
class _OrParams(C.Structure):
    _fields_ = [
        ("rho", C.c_double), ("nu", C.c_double), ("dt", C.c_double), ("ux", C.c_double),
        ("uz", C.c_double), ("cutoff_exp", C.c_double), ("max_numpanelvort", C.c_uint),
        ("scheme", C.c_int), ("surface_cross", C.c_int), ("seed", C.c_int),
    ]


class Port:
    """The C restatement (oracle/dvm_oracle.c)."""

    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        L = self.lib = C.CDLL(path)
        L.or_direct_self.argtypes = [_dp] * 4 + [C.c_size_t, _dp, _dp]
        L.or_direct_at.argtypes = [_dp] * 4 + [C.c_size_t, _dp, _dp, C.c_size_t, _dp, _dp]
        L.or_sheet_geometry.argtypes = [_dp, _dp, C.c_int] + [_dp] * 8
        L.or_influence_matrix.argtypes = [_dp] * 6 + [C.c_int, _dp]
        L.or_sheet_rhs.argtypes = [_dp] * 4 + [C.c_int, C.c_double, C.c_double] + [_dp] * 4 + [C.c_size_t, _dp]
        L.or_sheet_solve.argtypes = [_dp, _dp, C.c_int, _dp]
        L.or_sheet_on_blobs.argtypes = [_dp] * 5 + [C.c_int, _dp, _dp, C.c_size_t, _dp, _dp]
        L.or_diffuse.argtypes = [_dp, _dp, C.c_size_t, _dp, C.c_double, C.c_double]
        L.or_release_counts.argtypes = [_dp, _dp, C.c_int, C.c_uint, _dp, _dp]
        L.or_release_counts.restype = C.c_long
        L.or_release_place.argtypes = [_dp] * 7 + [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp] + [_dp] * 4
        L.or_inside.argtypes = [_dp, _dp, C.c_int, C.c_double, C.c_double]
        L.or_reflect.argtypes = [_dp] * 4 + [C.c_int, _dp, _dp, C.c_size_t]
        L.or_reflect.restype = C.c_size_t
        L.or_keep_flags.argtypes = [_dp, _dp, C.c_int, _dp, _dp, C.c_size_t, _u8p]
        L.or_keep_flags.restype = C.c_size_t
        L.or_loads.argtypes = [_dp] * 4 + [C.c_int] + [C.c_double] * 3 + [_dp, _dp]
        L.or_mt_stream.argtypes = [C.c_uint32, C.c_size_t, _dp]
        L.or_sim_create.argtypes = [C.POINTER(_OrParams), _dp, _dp, C.c_int]
        L.or_sim_create.restype = C.c_void_p
        L.or_sim_destroy.argtypes = [C.c_void_p]
        L.or_sim_set_blobs.argtypes = [C.c_void_p, C.c_size_t] + [_dp] * 4
        L.or_sim_step.argtypes = [C.c_void_p]
        L.or_sim_phase.argtypes = [C.c_void_p, C.c_int]
        L.or_sim_nblobs.argtypes = [C.c_void_p]
        L.or_sim_nblobs.restype = C.c_size_t
        L.or_sim_npanels.argtypes = [C.c_void_p]
        L.or_sim_get_blobs.argtypes = [C.c_void_p] + [_dp] * 8 + [_up]
        L.or_sim_get_sheet.argtypes = [C.c_void_p, _dp]
        L.or_sim_get_forces.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.or_sim_infm.argtypes = [C.c_void_p]
        L.or_sim_infm.restype = _dp

    # ---- kernels
    def direct_self(self, x, z, circ, sigma):
        x, z, circ, sigma = map(_f64, (x, z, circ, sigma))
        n = x.size
        u, w = np.empty(n), np.empty(n)
        self.lib.or_direct_self(_ptr(x), _ptr(z), _ptr(circ), _ptr(sigma), n, _ptr(u), _ptr(w))
        return u, w

    def direct_at(self, x, z, circ, sigma, tx, tz):
        x, z, circ, sigma, tx, tz = map(_f64, (x, z, circ, sigma, tx, tz))
        u, w = np.empty(tx.size), np.empty(tx.size)
        self.lib.or_direct_at(_ptr(x), _ptr(z), _ptr(circ), _ptr(sigma), x.size, _ptr(tx), _ptr(tz),
                              tx.size, _ptr(u), _ptr(w))
        return u, w

    def sheet_geometry(self, xp, zp):
        xp, zp = _f64(xp), _f64(zp)
        np_ = xp.size - 1
        out = [np.empty(np_) for _ in range(8)]
        self.lib.or_sheet_geometry(_ptr(xp), _ptr(zp), np_, *[_ptr(a) for a in out])
        keys = ["xc", "zc", "ds", "theta", "enx", "enz", "etx", "etz"]
        return dict(zip(keys, out))

    def influence_matrix(self, xp, zp):
        xp, zp = _f64(xp), _f64(zp)
        g = self.sheet_geometry(xp, zp)
        np_ = xp.size - 1
        A = np.empty((np_, np_ + 1))  # column-major (np+1) x np == row-major np x (np+1)
        self.lib.or_influence_matrix(_ptr(xp), _ptr(zp), _ptr(g["xc"]), _ptr(g["zc"]), _ptr(g["ds"]),
                                     _ptr(g["theta"]), np_, _ptr(A))
        return A.T.copy()

    def sheet_rhs(self, geo, Ux, Uz, x, z, circ, sigma):
        x, z, circ, sigma = map(_f64, (x, z, circ, sigma))
        np_ = geo["xc"].size
        b = np.empty(np_ + 1)
        self.lib.or_sheet_rhs(_ptr(geo["xc"]), _ptr(geo["zc"]), _ptr(geo["enx"]), _ptr(geo["enz"]), np_,
                              Ux, Uz, _ptr(x), _ptr(z), _ptr(circ), _ptr(sigma), x.size, _ptr(b))
        return b

    def sheet_solve(self, A, b):
        A = np.asfortranarray(A, dtype=np.float64)
        b = _f64(b)
        np_ = A.shape[1]
        g = np.empty(np_)
        Acm = np.ascontiguousarray(A.T)  # column-major buffer
        rc = self.lib.or_sheet_solve(_ptr(Acm), _ptr(b), np_, _ptr(g))
        if rc:
            raise RuntimeError("singular normal equations")
        return g

    def sheet_on_blobs(self, geo, gamma, x, z):
        x, z, gamma = _f64(x), _f64(z), _f64(gamma)
        np_ = gamma.size
        u, w = np.empty(x.size), np.empty(x.size)
        self.lib.or_sheet_on_blobs(_ptr(geo["xc"]), _ptr(geo["zc"]), _ptr(geo["theta"]), _ptr(geo["ds"]),
                                   _ptr(gamma), np_, _ptr(x), _ptr(z), x.size, _ptr(u), _ptr(w))
        return u, w

    def diffuse(self, x, z, R, nu, dt):
        x, z, R = _f64(x).copy(), _f64(z).copy(), _f64(R)
        assert R.size >= 2 * x.size
        self.lib.or_diffuse(_ptr(x), _ptr(z), x.size, _ptr(R), nu, dt)
        return x, z

    def release(self, xp, zp, gamma, M, nu, dt, cutoff_exp, R):
        xp, zp, gamma = _f64(xp), _f64(zp), _f64(gamma)
        g = self.sheet_geometry(xp, zp)
        np_ = gamma.size
        counts, cn = np.empty(np_), np.empty(np_)
        nrv = self.lib.or_release_counts(_ptr(gamma), _ptr(g["ds"]), np_, M, _ptr(counts), _ptr(cn))
        if nrv < 0:
            raise RuntimeError("release: negative PanelNewVort")
        R = _f64(R)
        assert R.size >= nrv
        out = [np.empty(nrv) for _ in range(4)]
        self.lib.or_release_place(_ptr(xp), _ptr(zp), _ptr(g["ds"]), _ptr(g["etx"]), _ptr(g["etz"]),
                                  _ptr(g["enx"]), _ptr(g["enz"]), np_, _ptr(counts), _ptr(cn), nu, dt,
                                  cutoff_exp, _ptr(R), *[_ptr(a) for a in out])
        return counts, out

    def inside(self, xp, zp, x, z):
        xp, zp = _f64(xp), _f64(zp)
        return np.array([self.lib.or_inside(_ptr(xp), _ptr(zp), xp.size - 1, float(a), float(b))
                         for a, b in zip(np.atleast_1d(x), np.atleast_1d(z))], dtype=np.uint8)

    def keep_flags(self, xp, zp, x, z):
        xp, zp, x, z = map(_f64, (xp, zp, x, z))
        keep = np.empty(x.size, dtype=np.uint8)
        self.lib.or_keep_flags(_ptr(xp), _ptr(zp), xp.size - 1, _ptr(x), _ptr(z), x.size, _ptr(keep))
        return keep

    def reflect(self, xp, zp, x, z):
        xp, zp = _f64(xp), _f64(zp)
        x, z = _f64(x).copy(), _f64(z).copy()
        g = self.sheet_geometry(xp, zp)
        moved = self.lib.or_reflect(_ptr(xp), _ptr(zp), _ptr(g["enx"]), _ptr(g["enz"]), xp.size - 1,
                                    _ptr(x), _ptr(z), x.size)
        return x, z, moved

    def loads(self, gamma, geo, rho, dt, Ur):
        gamma = _f64(gamma)
        fx, fz = C.c_double(), C.c_double()
        self.lib.or_loads(_ptr(gamma), _ptr(geo["ds"]), _ptr(geo["enx"]), _ptr(geo["enz"]), gamma.size,
                          rho, dt, Ur, C.byref(fx), C.byref(fz))
        return fx.value, fz.value

    def remesh(self, x, z, circ, sigma, x0, z0, dx, dz, nx, nz, kernel, new_sigma, threshold):
        x, z, circ, sigma = map(_f64, (x, z, circ, sigma))
        cap = nx * nz + x.size
        out = [np.empty(max(cap, 1)) for _ in range(4)]
        f = self.lib.or_remesh
        f.restype = C.c_size_t
        m = f(_ptr(x), _ptr(z), _ptr(circ), _ptr(sigma), C.c_size_t(x.size), C.c_double(x0),
              C.c_double(z0), C.c_double(dx), C.c_double(dz), C.c_int(nx), C.c_int(nz),
              C.c_int(kernel), C.c_double(new_sigma), C.c_double(threshold),
              *[_ptr(a) for a in out], C.c_size_t(cap))
        return [a[:m].copy() for a in out]

    def merge_blobs(self, d, threshold):
        """d: dict of x z circ sigma u w uvs wvs id; returns (new dict, merge count)."""
        keys = ["x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"]
        arrs = [np.array(d[k], dtype=np.float64) for k in keys]
        ids = np.array(d["id"], dtype=np.uint32)
        n_out = C.c_size_t()
        f = self.lib.or_merge_blobs
        f.restype = C.c_uint
        cnt = f(*[_ptr(a) for a in arrs], ids.ctypes.data_as(C.POINTER(C.c_uint)),
                C.c_size_t(ids.size), C.c_double(threshold), C.byref(n_out))
        m = n_out.value
        out = {k: a[:m].copy() for k, a in zip(keys, arrs)}
        out["id"] = ids[:m].copy()
        return out, int(cnt)

    def mt_stream(self, seed, n):
        out = np.empty(n)
        self.lib.or_mt_stream(seed, n, _ptr(out))
        return out

    # ---- whole simulation
    def sim(self, params: SimParams, xp, zp) -> "PortSim":
        return PortSim(self, params, xp, zp)


class PortSim:
    def __init__(self, port: Port, p: SimParams, xp, zp):
        self.L = port.lib
        xp, zp = _f64(xp), _f64(zp)
        cp = _OrParams(p.rho, p.nu, p.dt, p.ux, p.uz, p.cutoff_exp, p.max_numpanelvort, p.scheme_id(),
                       p.cross_id(), p.seed)
        self.h = self.L.or_sim_create(C.byref(cp), _ptr(xp), _ptr(zp), xp.size)
        self.np = xp.size - 1

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_sim_destroy(self.h)
            self.h = None

    def set_blobs(self, x, z, circ, sigma):
        x, z, circ, sigma = map(_f64, (x, z, circ, sigma))
        self.L.or_sim_set_blobs(self.h, x.size, _ptr(x), _ptr(z), _ptr(circ), _ptr(sigma))

    def step(self, n=1):
        for _ in range(n):
            if self.L.or_sim_step(self.h):
                raise RuntimeError("release threw (negative PanelNewVort)")

    def phase(self, k):
        rc = self.L.or_sim_phase(self.h, k)
        if rc:
            raise RuntimeError(f"phase {k} failed rc={rc}")

    @property
    def n(self):
        return self.L.or_sim_nblobs(self.h)

    def blobs(self):
        n = self.n
        arrs = [np.empty(n) for _ in range(8)]
        ids = np.empty(n, dtype=np.uint32)
        self.L.or_sim_get_blobs(self.h, *[_ptr(a) for a in arrs], _ptr(ids))
        keys = ["x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"]
        d = dict(zip(keys, arrs))
        d["id"] = ids
        return d

    def gamma(self):
        g = np.empty(self.np)
        self.L.or_sim_get_sheet(self.h, _ptr(g))
        return g

    def forces(self):
        fx, fz, a = C.c_double(), C.c_double(), C.c_double()
        self.L.or_sim_get_forces(self.h, C.byref(fx), C.byref(fz), C.byref(a))
        return fx.value, fz.value, a.value


# --------------------------------------------------------------------------
# The reference itself
# --------------------------------------------------------------------------
def write_case(directory: str, p: SimParams, xp, zp, stamp: str = "case") -> str:
    """Write a DVMpp XML input + body file (format of tests/fixtures in the
    reference: cylinder_test.xml, simple_body.txt).  Returns the XML path."""
    os.makedirs(directory, exist_ok=True)
    body = os.path.join(directory, "body.txt")
    with open(body, "w") as f:
        for a, b in zip(xp, zp):
            f.write(f"{a:.17g} {b:.17g}\n")
    xml = os.path.join(directory, stamp + ".xml")
    with open(xml, "w") as f:
        f.write(f"""<?xml version="1.0"?>
<DVMpp>
    <algorithms>
        <surface_crossing string="{p.surface_cross}" />
    </algorithms>
    <constants>
        <density val="{p.rho:.17g}" />
        <nu val="{p.nu:.17g}" />
        <max_NumPanelVort val="{p.max_numpanelvort}" />
        <cutoff_exp val="{p.cutoff_exp:.17g}" />
        <seed val="{p.seed}" />
    </constants>
    <io>
        <input_dir string="{directory}/" />
        <output_dir string="{directory}/" />
        <domain_file string="body.txt" />
    </io>
    <flow>
        <ux val="{p.ux:.17g}" />
        <uz val="{p.uz:.17g}" />
    </flow>
    <probe>
        <x val="20" />
        <z val="1" />
    </probe>
    <time>
        <scheme string="{p.scheme}" />
        <dt val="{p.dt:.17g}" />
        <steps val="{p.steps}" />
    </time>
</DVMpp>
""")
    return xml


class Ref:
    """The reference's own code (oracle/_ref/libdvmref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is")
        L = self.lib = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_direct_self.argtypes = [_dp] * 4 + [C.c_size_t, _dp, _dp]
        L.ref_direct_at.argtypes = [_dp] * 4 + [C.c_size_t, _dp, _dp, C.c_size_t, _dp, _dp]
        L.ref_random_stream.argtypes = [C.c_int, C.c_size_t, _dp]
        L.ref_sim_create.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.ref_sim_create.restype = C.c_void_p
        L.ref_sim_destroy.argtypes = [C.c_void_p]
        L.ref_sim_step.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.ref_sim_phase.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.ref_sim_nblobs.argtypes = [C.c_void_p]
        L.ref_sim_nblobs.restype = C.c_size_t
        L.ref_sim_write.argtypes = [C.c_void_p]
        L.ref_sim_npanels.argtypes = [C.c_void_p]
        L.ref_sim_get_blobs.argtypes = [C.c_void_p] + [_dp] * 8 + [_up]
        L.ref_sim_set_blobs.argtypes = [C.c_void_p, C.c_size_t] + [_dp] * 4
        L.ref_sim_get_sheet.argtypes = [C.c_void_p] + [_dp] * 9
        L.ref_sim_set_gamma.argtypes = [C.c_void_p, _dp]
        L.ref_sim_get_infm.argtypes = [C.c_void_p, _dp]
        L.ref_sim_get_forces.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.ref_sim_inside.argtypes = [C.c_void_p, C.c_double, C.c_double]

    def err(self):
        return self.lib.ref_last_error().decode()

    def direct_self(self, x, z, circ, sigma):
        x, z, circ, sigma = map(_f64, (x, z, circ, sigma))
        u, w = np.empty(x.size), np.empty(x.size)
        if self.lib.ref_direct_self(_ptr(x), _ptr(z), _ptr(circ), _ptr(sigma), x.size, _ptr(u), _ptr(w)):
            raise RuntimeError(self.err())
        return u, w

    def direct_at(self, x, z, circ, sigma, tx, tz):
        x, z, circ, sigma, tx, tz = map(_f64, (x, z, circ, sigma, tx, tz))
        u, w = np.empty(tx.size), np.empty(tx.size)
        if self.lib.ref_direct_at(_ptr(x), _ptr(z), _ptr(circ), _ptr(sigma), x.size, _ptr(tx), _ptr(tz),
                                  tx.size, _ptr(u), _ptr(w)):
            raise RuntimeError(self.err())
        return u, w

    def merge_blobs(self, d, threshold):
        keys = ["x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"]
        arrs = [np.array(d[k], dtype=np.float64) for k in keys]
        ids = np.array(d["id"], dtype=np.uint32)
        n_out, cnt = C.c_size_t(), C.c_uint()
        if self.lib.ref_merge_blobs(*[_ptr(a) for a in arrs],
                                    ids.ctypes.data_as(C.POINTER(C.c_uint)), C.c_size_t(ids.size),
                                    C.c_double(threshold), C.byref(n_out), C.byref(cnt)):
            raise RuntimeError(self.err())
        m = n_out.value
        out = {k: a[:m].copy() for k, a in zip(keys, arrs)}
        out["id"] = ids[:m].copy()
        return out, int(cnt.value)

    def random_stream(self, seed, n):
        out = np.empty(n)
        self.lib.ref_random_stream(seed, n, _ptr(out))
        return out

    def sim(self, params: SimParams, xp, zp, workdir: str | None = None, quiet=True) -> "RefSim":
        return RefSim(self, params, xp, zp, workdir, quiet)


class RefSim:
    def __init__(self, ref: Ref, p: SimParams, xp, zp, workdir=None, quiet=True):
        self.L = ref.lib
        self.ref = ref
        self.quiet = 1 if quiet else 0
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="dvmref_")
            workdir = self._tmp.name
        xml = write_case(workdir, p, xp, zp)
        self.h = self.L.ref_sim_create(xml.encode(), b"ref", self.quiet)
        if not self.h:
            raise RuntimeError(ref.err())
        self.np = self.L.ref_sim_npanels(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_sim_destroy(self.h)
            self.h = None

    def set_blobs(self, x, z, circ, sigma):
        x, z, circ, sigma = map(_f64, (x, z, circ, sigma))
        self.L.ref_sim_set_blobs(self.h, x.size, _ptr(x), _ptr(z), _ptr(circ), _ptr(sigma))

    def step(self, n=1):
        if self.L.ref_sim_step(self.h, n, self.quiet):
            raise RuntimeError(self.ref.err())

    def phase(self, k):
        if self.L.ref_sim_phase(self.h, k, self.quiet):
            raise RuntimeError(self.ref.err())

    def write_outputs(self):
        if self.L.ref_sim_write(self.h):
            raise RuntimeError(self.ref.err())

    @property
    def n(self):
        return self.L.ref_sim_nblobs(self.h)

    def blobs(self):
        n = self.n
        arrs = [np.empty(n) for _ in range(8)]
        ids = np.empty(n, dtype=np.uint32)
        self.L.ref_sim_get_blobs(self.h, *[_ptr(a) for a in arrs], _ptr(ids))
        keys = ["x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"]
        d = dict(zip(keys, arrs))
        d["id"] = ids
        return d

    def sheet(self):
        n = self.np
        arrs = [np.empty(n) for _ in range(7)] + [np.empty(n + 1), np.empty(n + 1)]
        self.L.ref_sim_get_sheet(self.h, *[_ptr(a) for a in arrs])
        keys = ["gamma", "xc", "zc", "ds", "theta", "enx", "enz", "x", "z"]
        return dict(zip(keys, arrs))

    def gamma(self):
        return self.sheet()["gamma"]

    def set_gamma(self, g):
        g = _f64(g)
        self.L.ref_sim_set_gamma(self.h, _ptr(g))

    def infm(self):
        A = np.empty((self.np, self.np + 1))
        self.L.ref_sim_get_infm(self.h, _ptr(A))
        return A.T.copy()

    def forces(self):
        fx, fz, a = C.c_double(), C.c_double(), C.c_double()
        self.L.ref_sim_get_forces(self.h, C.byref(fx), C.byref(fz), C.byref(a))
        return fx.value, fz.value, a.value


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def have_port() -> bool:
    return os.path.exists(PORT_SO)
