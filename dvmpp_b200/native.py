"""ctypes binding of the C ABI in include/dvm_cuda.h (libdvm_cuda.so).

This is the Python face of the drop-in boundary: it calls exactly the entry
points a cgo / JNI / ctypes user would bind.  There is no fallback: if the
CUDA library is missing, or no B200 is visible, every call raises.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DVMPP_CUDA_LIB") or os.path.join(HERE, "lib", "libdvm_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "dvm_cuda.h")

OK, ERR_ARG, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_CAPACITY, ERR_RELEASE, ERR_STATE, ERR_RNG, ERR_NO_DEVICE = range(10)
F64, F32 = 0, 1
EULER, RK3 = 0, 1
DELETE, ABSORB, REFLECT = 0, 1, 2
RNG_INJECT, RNG_PHILOX = 0, 1
PROF_FAMILIES = ["nbody", "rhs", "solve", "sheetvel", "diffuse_release", "cross", "loads", "sort",
                 "step"]
(PHASE_BIOTSAVART, PHASE_SOLVE, PHASE_SHEETBC, PHASE_CONVECT, PHASE_DIFFUSE, PHASE_RELEASE,
 PHASE_CROSS, PHASE_LOADS, PHASE_INCREMENT, PHASE_REFLECT, PHASE_DELETE) = range(11)

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)


class DvmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class Particle(C.Structure):
    _fields_ = [("x", C.c_double), ("z", C.c_double), ("circ", C.c_double), ("sigma", C.c_double)]


class Velocity(C.Structure):
    _fields_ = [("u", C.c_double), ("w", C.c_double)]


class SimParams(C.Structure):
    _fields_ = [
        ("rho", C.c_double), ("nu", C.c_double), ("dt", C.c_double), ("ux", C.c_double),
        ("uz", C.c_double), ("cutoff_exp", C.c_double), ("max_numpanelvort", C.c_uint32),
        ("scheme", C.c_int32), ("surface_cross", C.c_int32), ("rng", C.c_int32),
        ("precision", C.c_int32), ("reserved", C.c_int32), ("seed", C.c_int64),
        ("capacity", C.c_uint64), ("rng_capacity", C.c_uint64),
    ]


# name -> (restype, argtypes); every symbol declared in include/dvm_cuda.h
SIGNATURES = {
    "dvm_abi_version": (C.c_int, []),
    "dvm_status_string": (C.c_char_p, [C.c_int]),
    "dvm_last_error": (C.c_char_p, []),
    "dvm_ctx_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "dvm_ctx_destroy": (C.c_int, [C.c_void_p]),
    "dvm_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "dvm_ctx_memory": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "dvm_ctx_device_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "dvm_ctx_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "dvm_sim_bytes": (C.c_int, [C.POINTER(SimParams), C.c_int, C.POINTER(C.c_uint64)]),
    "dvm_ctx_mark": (C.c_int, [C.c_void_p, C.c_int]),
    "dvm_ctx_elapsed": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
    "dvm_ctx_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "dvm_ctx_profiler_range": (C.c_int, [C.c_void_p, C.c_int]),
    "dvm_ctx_profile": (C.c_int, [C.c_void_p, C.c_int, _dp, C.POINTER(C.c_uint64)]),
    "dvm_ctx_profile_reset": (C.c_int, [C.c_void_p]),
    "dvm_biot_savart_self": (C.c_int, [C.c_void_p, C.POINTER(Particle), C.c_uint64, C.POINTER(Velocity), C.c_int]),
    "dvm_biot_savart_at": (C.c_int, [C.c_void_p, C.POINTER(Particle), C.c_uint64, _dp, _dp, C.c_uint64,
                                     C.POINTER(Velocity), C.c_int]),
    "dvm_biot_savart_self_device": (C.c_int, [C.c_void_p] + [C.c_void_p] * 4 + [C.c_uint64] + [C.c_void_p] * 2 + [C.c_int]),
    "dvm_biot_savart_at_device": (C.c_int, [C.c_void_p] + [C.c_void_p] * 4 + [C.c_uint64] + [C.c_void_p] * 2
                                  + [C.c_uint64] + [C.c_void_p] * 2 + [C.c_int, C.c_int]),
    "dvm_biot_savart_at_noalloc": (C.c_int, [C.c_void_p] * 4 + [C.c_uint64] + [C.c_void_p] * 2
                                   + [C.c_uint64] + [C.c_void_p] * 2 + [C.c_int, C.c_int, C.c_void_p]),
    "dvm_sim_create": (C.c_int, [C.c_void_p, C.POINTER(SimParams), _dp, _dp, C.c_int, C.POINTER(C.c_void_p)]),
    "dvm_sims_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.POINTER(SimParams)), C.POINTER(_dp),
                                  C.POINTER(_dp), C.POINTER(C.c_int), C.POINTER(C.c_void_p)]),
    "dvm_sim_destroy": (C.c_int, [C.c_void_p]),
    "dvm_sim_set_blobs": (C.c_int, [C.c_void_p, C.c_uint64, _dp, _dp, _dp, _dp]),
    "dvm_sim_get_blobs": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)] + [_dp] * 8 + [_u32p]),
    "dvm_sim_num_blobs": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "dvm_sim_num_panels": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "dvm_sim_get_gamma": (C.c_int, [C.c_void_p, _dp]),
    "dvm_sim_set_gamma": (C.c_int, [C.c_void_p, _dp]),
    "dvm_sim_get_rhs": (C.c_int, [C.c_void_p, _dp]),
    "dvm_sim_get_influence": (C.c_int, [C.c_void_p, _dp]),
    "dvm_sim_get_panels": (C.c_int, [C.c_void_p] + [_dp] * 6),
    "dvm_sim_get_loads": (C.c_int, [C.c_void_p] + [_dp] * 4),
    "dvm_sim_get_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "dvm_sim_push_uniforms": (C.c_int, [C.c_void_p, _dp, C.c_uint64]),
    "dvm_sim_rng_position": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "dvm_sim_status": (C.c_int, [C.c_void_p]),
    "dvm_sim_clear_status": (C.c_int, [C.c_void_p]),
    "dvm_sim_phase": (C.c_int, [C.c_void_p, C.c_int]),
    "dvm_sim_step": (C.c_int, [C.c_void_p, C.c_int]),
    "dvm_step_batch": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int]),
}

_LIB = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libdvm_cuda.so (raises if it is absent: there is no CPU path)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing; build it with `python -m dvmpp_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


def _check(rc: int):
    if rc != OK:
        raise DvmError(rc, _LIB.dvm_last_error().decode(errors="replace"))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


class Context:
    """One device, one stream, an HBM budget (dvm_ctx)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        self.lib = load()
        h = C.c_void_p()
        _check(self.lib.dvm_ctx_create(device, budget_bytes, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.dvm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sync(self):
        _check(self.lib.dvm_ctx_synchronize(self.h))

    def memory(self):
        a, b = C.c_uint64(), C.c_uint64()
        _check(self.lib.dvm_ctx_memory(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def reserve(self, total_capacity: int, max_sims: int, max_panels: int, with_delete=False):
        """Pre-size the shared workspace for batches up to these sizes."""
        _check(self.lib.dvm_ctx_reserve(self.h, int(total_capacity), int(max_sims),
                                        int(max_panels), 1 if with_delete else 0))

    def pool_reserve(self, nbytes: int):
        """Map the stream-ordered pool for simulation slabs up to nbytes once."""
        _check(self.lib.dvm_ctx_pool_reserve(self.h, int(nbytes)))

    def device_info(self):
        s, ma, mi = C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.dvm_ctx_device_info(self.h, C.byref(s), C.byref(ma), C.byref(mi)))
        return s.value, ma.value, mi.value

    def mark(self, slot: int):
        _check(self.lib.dvm_ctx_mark(self.h, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        v = C.c_double()
        _check(self.lib.dvm_ctx_elapsed(self.h, a, b, C.byref(v)))
        return v.value

    def profiler_range(self, on: bool):
        _check(self.lib.dvm_ctx_profiler_range(self.h, 1 if on else 0))

    def set_profiling(self, on: bool):
        _check(self.lib.dvm_ctx_set_profiling(self.h, 1 if on else 0))

    def profile(self):
        """{family: (total ms, timed launches)} from CUDA events on the ctx stream."""
        out = {}
        for k, name in enumerate(PROF_FAMILIES):
            ms, n = C.c_double(), C.c_uint64()
            _check(self.lib.dvm_ctx_profile(self.h, k, C.byref(ms), C.byref(n)))
            out[name] = (ms.value, n.value)
        return out

    def profile_reset(self):
        _check(self.lib.dvm_ctx_profile_reset(self.h))

    def launches(self) -> int:
        v = C.c_uint64()
        _check(self.lib.dvm_ctx_launch_count(self.h, C.byref(v)))
        return v.value

    # ---- VelocityKernel plugin seam
    def biot_savart_self(self, x, z, circ, sigma, precision=F32):
        n = len(x)
        p = (Particle * max(n, 1))()
        arr = np.frombuffer(p, dtype=np.float64, count=4 * n).reshape(n, 4) if n else None
        if n:
            arr[:, 0], arr[:, 1], arr[:, 2], arr[:, 3] = x, z, circ, sigma
        out = (Velocity * max(n, 1))()
        _check(self.lib.dvm_biot_savart_self(self.h, p, n, out, precision))
        v = np.frombuffer(out, dtype=np.float64, count=2 * n).reshape(n, 2) if n else np.zeros((0, 2))
        return v[:, 0].copy(), v[:, 1].copy()

    def biot_savart_at(self, x, z, circ, sigma, tx, tz, precision=F32):
        n = len(x)
        p = (Particle * max(n, 1))()
        if n:
            arr = np.frombuffer(p, dtype=np.float64, count=4 * n).reshape(n, 4)
            arr[:, 0], arr[:, 1], arr[:, 2], arr[:, 3] = x, z, circ, sigma
        tx, tz = _f64(tx), _f64(tz)
        nt = tx.size
        out = (Velocity * max(nt, 1))()
        _check(self.lib.dvm_biot_savart_at(self.h, p, n, _p(tx), _p(tz), nt, out, precision))
        v = np.frombuffer(out, dtype=np.float64, count=2 * nt).reshape(nt, 2) if nt else np.zeros((0, 2))
        return v[:, 0].copy(), v[:, 1].copy()

    def merge_blobs(self, d: dict, threshold: float):
        """Greedy merge on host arrays (the VortexBlobs::merge_blobs path).
        d: x z circ sigma u w uvs wvs (+ id); returns (new dict, merge count)."""
        keys = ["x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"]
        arrs = [np.array(d[k], dtype=np.float64) for k in keys]
        n = arrs[0].size
        ids = np.array(d.get("id", np.arange(n)), dtype=np.uint32)
        m, cnt = C.c_uint64(), C.c_uint64()
        _check(self.lib.dvm_merge_blobs(self.h, *[_p(a) for a in arrs],
                                        ids.ctypes.data_as(_u32p), n, threshold, C.byref(m),
                                        C.byref(cnt)))
        out = {k: a[:m.value].copy() for k, a in zip(keys, arrs)}
        out["id"] = ids[:m.value].copy()
        return out, cnt.value

    def remesh(self, x, z, circ, sigma, params: RemeshParams, out_cap=None):
        """Remesh host arrays (the BackgroundMesh::remesh path): (x, z, circ, sigma)."""
        n = len(x)
        p = (Particle * max(n, 1))()
        if n:
            arr = np.frombuffer(p, dtype=np.float64, count=4 * n).reshape(n, 4)
            arr[:, 0], arr[:, 1], arr[:, 2], arr[:, 3] = x, z, circ, sigma
        if out_cap is None:
            nx, nz = remesh_grid(params)
            out_cap = nx * nz + n
        out = (Particle * max(out_cap, 1))()
        m = C.c_uint64()
        _check(self.lib.dvm_remesh(self.h, p, n, C.byref(params), out, out_cap, C.byref(m)))
        v = np.frombuffer(out, dtype=np.float64, count=4 * m.value).reshape(m.value, 4)
        return tuple(v[:, k].copy() for k in range(4))

    def step_batch(self, sims, nsteps=1, use_graph=True):
        arr = (C.c_void_p * len(sims))(*[s.h for s in sims])
        _check(self.lib.dvm_step_batch(self.h, arr, len(sims), nsteps, 1 if use_graph else 0))

    # ---- pair-kernel autotuning
    @staticmethod
    def _sim_array(sims):
        return (C.c_void_p * len(sims))(*[s.h for s in sims])

    def autotune(self, sims, reps: int = 1) -> dict:
        """Time every pair-kernel launch shape on this batch and keep the best
        for its shape class; returns the candidates' times."""
        r = TuneResult()
        _check(self.lib.dvm_ctx_autotune(self.h, self._sim_array(sims), len(sims), reps,
                                         C.byref(r)))
        cands = tune_candidates()
        return {"shape_class": r.shape_class, "best": r.best.as_dict(), "best_ms": r.best_ms,
                "default_ms": r.default_ms,
                "candidates": [dict(c, ms=r.ms[k]) for k, c in enumerate(cands[:r.candidates])]}

    def batch_get_state(self, sims, xs=None, zs=None, cs=None):
        """Blob counts and loads of many simulations with one wait; x / z / circ
        copied into the given buffers (lists of float64 arrays, e.g. pinned).
        Returns (counts, loads[nsims, 4])."""
        n = len(sims)
        P = C.POINTER(C.c_double)

        def ptrs(bufs):
            return None if bufs is None else (P * n)(*[_p(b) for b in bufs])

        given = [arr for arr in (xs, zs, cs) if arr is not None]
        caps = (C.c_uint64 * n)(*[min(a[i].size for a in given) if given else 0
                                  for i in range(n)])
        counts = (C.c_uint64 * n)()
        loads = np.empty((n, 4))
        _check(self.lib.dvm_batch_get_state(self.h, self._sim_array(sims), n, ptrs(xs), ptrs(zs),
                                            ptrs(cs), caps, counts, _p(loads)))
        return [int(counts[i]) for i in range(n)], loads

    def batch_push_uniforms(self, sims, bufs, counts):
        n = len(sims)
        P = C.POINTER(C.c_double)
        arr = (P * n)(*[_p(b) for b in bufs])
        cnt = (C.c_uint64 * n)(*[int(k) for k in counts])
        _check(self.lib.dvm_batch_push_uniforms(self.h, self._sim_array(sims), n, arr, cnt))

    def batch_push_uniforms_async(self, sims, bufs, counts):
        """Append uniforms on the copy stream without waiting (bufs: pinned
        float64 arrays, unchanged until the next batch_wait_state); the next
        enqueued step waits for the copies.  Never compacts the stream."""
        n = len(sims)
        P = C.POINTER(C.c_double)
        arr = (P * n)(*[_p(b) for b in bufs])
        cnt = (C.c_uint64 * n)(*[int(k) for k in counts])
        _check(self.lib.dvm_batch_push_uniforms_async(self.h, self._sim_array(sims), n, arr, cnt))

    def batch_get_state_async(self, sims):
        """Snapshot the state of sims on the GPU after the enqueued work (no wait)."""
        self._snap_n = len(sims)
        _check(self.lib.dvm_batch_get_state_async(self.h, self._sim_array(sims), len(sims)))

    def batch_wait_state(self, xs=None, zs=None, cs=None):
        """Wait for the pending snapshot and copy it out (while later enqueued
        steps run).  Returns (counts, loads[nsims, 4])."""
        n = getattr(self, "_snap_n", 0)
        P = C.POINTER(C.c_double)

        def ptrs(bufs):
            return None if bufs is None else (P * n)(*[_p(b) for b in bufs])

        given = [arr for arr in (xs, zs, cs) if arr is not None]
        caps = (C.c_uint64 * max(n, 1))(*[min(a[i].size for a in given) if given else 0
                                          for i in range(n)])
        counts = (C.c_uint64 * max(n, 1))()
        loads = np.empty((n, 4))
        _check(self.lib.dvm_batch_wait_state(self.h, n, ptrs(xs), ptrs(zs), ptrs(cs), caps, counts,
                                             _p(loads)))
        return [int(counts[i]) for i in range(n)], loads

    def batch_status(self, sims) -> list:
        out = (C.c_int32 * max(len(sims), 1))()
        _check(self.lib.dvm_batch_status(self.h, self._sim_array(sims), len(sims), out))
        return [int(out[k]) for k in range(len(sims))]

    def shape_class(self, sims) -> int:
        v = C.c_int()
        _check(self.lib.dvm_batch_shape_class(self.h, self._sim_array(sims), len(sims),
                                              C.byref(v)))
        return v.value

    def set_pair_config(self, shape_class: int, tile: int, ctas_per_sm: int, order: int):
        cfg = PairConfig(tile, ctas_per_sm, order, 0)
        _check(self.lib.dvm_ctx_set_pair_config(self.h, shape_class, C.byref(cfg)))

    def pair_config(self, shape_class: int) -> dict:
        cfg = PairConfig()
        _check(self.lib.dvm_ctx_get_pair_config(self.h, shape_class, C.byref(cfg)))
        return cfg.as_dict()

    def tuning_table(self) -> dict:
        """{shape_class: config} of every tuned class."""
        n = C.c_int()
        _check(self.lib.dvm_ctx_tuning_table(self.h, 0, None, None, C.byref(n)))
        cls = (C.c_int * max(n.value, 1))()
        cfgs = (PairConfig * max(n.value, 1))()
        _check(self.lib.dvm_ctx_tuning_table(self.h, n.value, cls, cfgs, C.byref(n)))
        return {int(cls[k]): cfgs[k].as_dict() for k in range(n.value)}

    def save_tuning(self, path: str):
        with open(path, "w") as f:
            json.dump({str(k): v for k, v in self.tuning_table().items()}, f, indent=1)

    def load_tuning(self, path: str):
        with open(path) as f:
            for k, v in json.load(f).items():
                self.set_pair_config(int(k), v["tile"], v["ctas_per_sm"], v["order"])

    def sim(self, params: "Params", xp, zp) -> "Simulation":
        return Simulation(self, params, xp, zp)

    def sims(self, params, bodies) -> list:
        """Several simulations created together (dvm_sims_create): their bodies'
        factorisations share launches.  params: one Params per body; bodies:
        (x, z) contours.  All are created, or none (the error is raised)."""
        n = len(bodies)
        cps = [p.c() for p in params]
        xs = [_f64(x) for x, _ in bodies]
        zs = [_f64(z) for _, z in bodies]
        pp = (C.POINTER(SimParams) * n)(*[C.pointer(cp) for cp in cps])
        px = (_dp * n)(*[_p(x) for x in xs])
        pz = (_dp * n)(*[_p(z) for z in zs])
        npts = (C.c_int * n)(*[x.size for x in xs])
        hs = (C.c_void_p * n)()
        _check(self.lib.dvm_sims_create(self.h, n, pp, px, pz, npts, hs))
        out = []
        for k in range(n):
            sim = Simulation.__new__(Simulation)
            sim.ctx, sim.lib, sim.h = self, self.lib, C.c_void_p(hs[k])
            sim.params = params[k]
            sim.np = xs[k].size - 1
            out.append(sim)
        return out

    def restore(self, state: bytes, params: "Params" = None) -> "Simulation":
        """A simulation rebuilt from Simulation.save() output (in this context)."""
        h = C.c_void_p()
        buf = C.create_string_buffer(bytes(state), len(state))
        _check(self.lib.dvm_sim_restore(self.h, buf, len(state), C.byref(h)))
        sim = Simulation.__new__(Simulation)
        sim.ctx, sim.lib, sim.h = self, self.lib, h
        sim.params = params
        npn = C.c_int()
        _check(self.lib.dvm_sim_num_panels(h, C.byref(npn)))
        sim.np = npn.value
        return sim


@dataclass
class Params:
    rho: float = 1.0
    nu: float = 1e-3
    dt: float = 0.005
    ux: float = 3.0
    uz: float = 0.0
    cutoff_exp: float = 0.675
    max_numpanelvort: int = 3
    scheme: int = EULER
    surface_cross: int = REFLECT
    rng: int = RNG_INJECT
    precision: int = F64
    seed: int = 1
    capacity: int = 1 << 16
    rng_capacity: int = 1 << 20

    def c(self) -> SimParams:
        return SimParams(self.rho, self.nu, self.dt, self.ux, self.uz, self.cutoff_exp,
                         self.max_numpanelvort, self.scheme, self.surface_cross, self.rng,
                         self.precision, 0, self.seed, self.capacity, self.rng_capacity)


def sim_bytes(params: Params, npanels: int) -> int:
    lib = load()
    b = C.c_uint64()
    cp = params.c()
    _check(lib.dvm_sim_bytes(C.byref(cp), npanels, C.byref(b)))
    return b.value


class Simulation:
    """One simulation resident on the device (dvm_sim)."""

    def __init__(self, ctx: Context, params: Params, xp, zp):
        self.ctx = ctx
        self.lib = ctx.lib
        self.params = params
        xp, zp = _f64(xp), _f64(zp)
        h = C.c_void_p()
        cp = params.c()
        _check(self.lib.dvm_sim_create(ctx.h, C.byref(cp), _p(xp), _p(zp), xp.size, C.byref(h)))
        self.h = h
        self.np = xp.size - 1

    def close(self):
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            self.lib.dvm_sim_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def save(self) -> bytes:
        """Everything a later step depends on (dvm_sim_save), as bytes."""
        n = C.c_uint64()
        _check(self.lib.dvm_sim_state_size(self.h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        w = C.c_uint64()
        _check(self.lib.dvm_sim_save(self.h, buf, n.value, C.byref(w)))
        return buf.raw[:w.value]

    def set_blobs(self, x, z, circ, sigma):
        x, z, circ, sigma = map(_f64, (x, z, circ, sigma))
        _check(self.lib.dvm_sim_set_blobs(self.h, x.size, _p(x), _p(z), _p(circ), _p(sigma)))

    @property
    def n(self) -> int:
        v = C.c_uint64()
        _check(self.lib.dvm_sim_num_blobs(self.h, C.byref(v)))
        return v.value

    def blobs(self):
        n = self.n
        arrs = [np.empty(n) for _ in range(8)]
        ids = np.empty(n, dtype=np.uint32)
        nn = C.c_uint64()
        _check(self.lib.dvm_sim_get_blobs(self.h, n, C.byref(nn), *[_p(a) for a in arrs],
                                          ids.ctypes.data_as(_u32p)))
        d = dict(zip(["x", "z", "circ", "sigma", "u", "w", "uvs", "wvs"], arrs))
        d["id"] = ids
        return d

    def get_state_into(self, x, z, circ):
        """Copy positions and circulations into caller buffers (e.g. pinned);
        returns the blob count (also kept in self.last_n)."""
        nn = C.c_uint64()
        cap = min(x.size, z.size, circ.size)
        _check(self.lib.dvm_sim_get_blobs(self.h, cap, C.byref(nn), _p(x), _p(z), _p(circ),
                                          None, None, None, None, None, None))
        self.last_n = nn.value
        return nn.value

    def gamma(self):
        g = np.empty(self.np)
        _check(self.lib.dvm_sim_get_gamma(self.h, _p(g)))
        return g

    def set_gamma(self, g):
        g = _f64(g)
        _check(self.lib.dvm_sim_set_gamma(self.h, _p(g)))

    def rhs(self):
        b = np.empty(self.np + 1)
        _check(self.lib.dvm_sim_get_rhs(self.h, _p(b)))
        return b

    def influence(self):
        A = np.empty((self.np + 1, self.np))
        _check(self.lib.dvm_sim_get_influence(self.h, _p(A)))
        return A

    def panels(self):
        arrs = [np.empty(self.np) for _ in range(6)]
        _check(self.lib.dvm_sim_get_panels(self.h, *[_p(a) for a in arrs]))
        return dict(zip(["xc", "zc", "ds", "theta", "enx", "enz"], arrs))

    def loads(self):
        v = [C.c_double() for _ in range(4)]
        _check(self.lib.dvm_sim_get_loads(self.h, *[C.byref(a) for a in v]))
        return tuple(a.value for a in v)  # fx, fz, cd, cl

    def step_number(self) -> int:
        v = C.c_uint32()
        _check(self.lib.dvm_sim_get_step(self.h, C.byref(v)))
        return v.value

    def push_uniforms(self, u):
        u = _f64(u)
        _check(self.lib.dvm_sim_push_uniforms(self.h, _p(u), u.size))

    def rng_position(self):
        a, b = C.c_uint64(), C.c_uint64()
        _check(self.lib.dvm_sim_rng_position(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def status(self) -> int:
        return self.lib.dvm_sim_status(self.h)

    def check(self):
        _check(self.lib.dvm_sim_status(self.h))

    def merge(self, threshold: float) -> int:
        """Greedy vortex merge in place on the device; returns the merge count."""
        m = C.c_uint64()
        _check(self.lib.dvm_sim_merge(self.h, threshold, C.byref(m)))
        return m.value

    def remesh(self, params: "RemeshParams") -> int:
        """Remesh in place on the device; returns the new blob count."""
        n = C.c_uint64()
        _check(self.lib.dvm_sim_remesh(self.h, C.byref(params), C.byref(n)))
        return n.value

    def probe(self, px, pz):
        """Velocity at probe points: (u, w, uvs, wvs) with u, w the total."""
        px, pz = _f64(px), _f64(pz)
        n = px.size
        out = [np.empty(n) for _ in range(4)]
        _check(self.lib.dvm_sim_probe(self.h, _p(px), _p(pz), n, *[_p(a) for a in out]))
        return tuple(out)

    def clear_status(self):
        _check(self.lib.dvm_sim_clear_status(self.h))

    def phase(self, k: int):
        _check(self.lib.dvm_sim_phase(self.h, k))

    def step(self, nsteps: int = 1):
        _check(self.lib.dvm_sim_step(self.h, nsteps))


# ---- serving ----------------------------------------------------------------
SERVE_GRAPH, SERVE_SYNC, SERVE_AUTOTUNE, SERVE_LIVE = 0, 1, 2, 3


class RequestResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("arrival_s", C.c_double), ("admitted_s", C.c_double),
                ("finished_s", C.c_double), ("latency_s", C.c_double), ("steps_done", C.c_uint32),
                ("status", C.c_int32), ("blobs", C.c_uint64), ("fx", C.c_double),
                ("fz", C.c_double), ("cd", C.c_double), ("cl", C.c_double)]


class ServerSummary(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("sim_steps", C.c_uint64), ("ticks", C.c_uint64), ("wall_s", C.c_double),
                ("sim_steps_per_s", C.c_double), ("latency_p50_s", C.c_double),
                ("latency_p95_s", C.c_double), ("latency_p99_s", C.c_double),
                ("latency_mean_s", C.c_double), ("queue_p50_s", C.c_double),
                ("queue_p99_s", C.c_double), ("peak_active", C.c_uint32),
                ("peak_bytes", C.c_uint64), ("admit_s", C.c_double), ("step_s", C.c_double),
                ("retire_s", C.c_double), ("tunings", C.c_uint32)]


REMESH_M4PRIME, REMESH_M6, REMESH_GAUSSIAN = 0, 1, 2


class RemeshParams(C.Structure):
    _fields_ = [("xmin", C.c_double), ("xmax", C.c_double), ("zmin", C.c_double),
                ("zmax", C.c_double), ("dx", C.c_double), ("dz", C.c_double),
                ("sigma", C.c_double), ("circ_threshold", C.c_double), ("kernel", C.c_int32),
                ("reserved", C.c_int32)]


def remesh_grid(params: RemeshParams):
    nx, nz = C.c_uint32(), C.c_uint32()
    _check(load().dvm_remesh_grid(C.byref(params), C.byref(nx), C.byref(nz)))
    return nx.value, nz.value


class PairConfig(C.Structure):
    _fields_ = [("tile", C.c_int32), ("ctas_per_sm", C.c_int32), ("order", C.c_int32),
                ("reserved", C.c_int32)]

    def as_dict(self):
        return {"tile": self.tile, "ctas_per_sm": self.ctas_per_sm, "order": self.order}


TUNE_MAX_CANDIDATES = 16


class TuneResult(C.Structure):
    _fields_ = [("best", PairConfig), ("shape_class", C.c_int32), ("candidates", C.c_int32),
                ("best_ms", C.c_double), ("default_ms", C.c_double),
                ("ms", C.c_double * TUNE_MAX_CANDIDATES)]


def philox4x32_10(ctr, key):
    """The device Philox4x32-10 on blocks: ctr (n, 4) and key (n, 2) uint32
    arrays -> (n, 4) outputs."""
    lib = load()
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, dtype=np.uint32).reshape(-1, 2)
    if ctr.shape[0] != key.shape[0]:
        raise ValueError("ctr and key must have the same number of blocks")
    out = np.empty_like(ctr)
    _check(lib.dvm_philox4x32_10(ctr.ctypes.data_as(_u32p), key.ctypes.data_as(_u32p), ctr.shape[0],
                                 out.ctypes.data_as(_u32p)))
    return out


def tune_candidates() -> list:
    """The autotuner's search space, in the order it times it."""
    lib = load()
    out, k = [], 0
    cfg = PairConfig()
    while lib.dvm_tune_candidate(k, C.byref(cfg)) == OK:
        out.append(cfg.as_dict())
        k += 1
    return out


SIGNATURES.update({
    "dvm_tune_candidate": (C.c_int, [C.c_int, C.POINTER(PairConfig)]),
    "dvm_ctx_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(TuneResult)]),
    "dvm_batch_shape_class": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "dvm_ctx_set_pair_config": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(PairConfig)]),
    "dvm_ctx_get_pair_config": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(PairConfig)]),
    "dvm_ctx_tuning_table": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(PairConfig), C.POINTER(C.c_int)]),
    "dvm_batch_status": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int32)]),
    "dvm_batch_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                      _dp]),
    "dvm_batch_push_uniforms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.POINTER(C.c_uint64)]),
    "dvm_batch_push_uniforms_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                                C.POINTER(C.c_uint64)]),
    "dvm_batch_get_state_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "dvm_batch_wait_state": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _dp]),
    "dvm_sim_probe": (C.c_int, [C.c_void_p, _dp, _dp, C.c_uint64, _dp, _dp, _dp, _dp]),
    "dvm_sim_merge": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_uint64)]),
    "dvm_merge_blobs": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _u32p,
                                  C.c_uint64, C.c_double, C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint64)]),
    "dvm_remesh_grid": (C.c_int, [C.POINTER(RemeshParams), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32)]),
    "dvm_sim_remesh": (C.c_int, [C.c_void_p, C.POINTER(RemeshParams), C.POINTER(C.c_uint64)]),
    "dvm_remesh": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(RemeshParams),
                             C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
})


SIGNATURES.update({
    "dvm_ctx_reserve": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int]),
    "dvm_random_walk": (C.c_int, [C.c_void_p, _dp, _dp, C.c_uint64, _dp, C.c_double, C.c_double]),
    "dvm_philox4x32_10": (C.c_int, [_u32p, _u32p, C.c_uint64, _u32p]),
    "dvm_sim_set_step": (C.c_int, [C.c_void_p, C.c_uint32]),
    "dvm_sim_state_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "dvm_sim_save": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "dvm_sim_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_void_p)]),
    "dvm_sim_clear_uniforms": (C.c_int, [C.c_void_p]),
    "dvm_sim_pending_uniforms": (C.c_int, [C.c_void_p, _dp, C.c_uint64, C.POINTER(C.c_uint64)]),
    "dvm_ctx_workspace_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "dvm_ctx_pool_reserve": (C.c_int, [C.c_void_p, C.c_uint64]),
    "dvm_server_create": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "dvm_server_destroy": (C.c_int, [C.c_void_p]),
    "dvm_server_set_option": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dvm_server_submit": (C.c_int, [C.c_void_p, C.POINTER(SimParams), _dp, _dp, C.c_int, C.c_uint32,
                                    C.c_double, C.POINTER(C.c_uint64)]),
    "dvm_server_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dvm_server_close_intake": (C.c_int, [C.c_void_p]),
    "dvm_server_result": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(RequestResult)]),
    "dvm_server_final_blobs": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64),
                                         _dp, _dp, _dp]),
    "dvm_server_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerSummary)]),
})


class Server:
    """Continuous-batching request loop over one Context (dvm_server)."""

    def __init__(self, ctx: Context, budget_bytes: int = 0, max_active: int = 64, keep_state=False):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        _check(self.lib.dvm_server_create(ctx.h, budget_bytes, max_active, 1 if keep_state else 0,
                                          C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            self.lib.dvm_server_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def set_option(self, option: int, value: int):
        _check(self.lib.dvm_server_set_option(self.h, option, value))

    def submit(self, params: Params, xp, zp, steps: int, arrival_s: float = -1.0) -> int:
        """arrival_s < 0: the request arrives when submitted."""
        xp, zp = _f64(xp), _f64(zp)
        cp = params.c()
        rid = C.c_uint64()
        _check(self.lib.dvm_server_submit(self.h, C.byref(cp), _p(xp), _p(zp), xp.size, steps,
                                          arrival_s, C.byref(rid)))
        return rid.value

    def run(self, serial=False, realtime=False):
        """Blocks until the run ends (ctypes releases the GIL meanwhile, so
        other Python threads may submit)."""
        _check(self.lib.dvm_server_run(self.h, 1 if serial else 0, 1 if realtime else 0))

    def close_intake(self):
        _check(self.lib.dvm_server_close_intake(self.h))

    def result(self, rid: int) -> dict:
        r = RequestResult()
        _check(self.lib.dvm_server_result(self.h, rid, C.byref(r)))
        return {f: getattr(r, f) for f, _ in RequestResult._fields_}

    def final_blobs(self, rid: int):
        n = C.c_uint64()
        _check(self.lib.dvm_server_final_blobs(self.h, rid, 0, C.byref(n), None, None, None))
        x, z, c = np.empty(n.value), np.empty(n.value), np.empty(n.value)
        _check(self.lib.dvm_server_final_blobs(self.h, rid, n.value, C.byref(n), _p(x), _p(z), _p(c)))
        return x, z, c

    def stats(self) -> dict:
        s = ServerSummary()
        _check(self.lib.dvm_server_stats(self.h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerSummary._fields_}
