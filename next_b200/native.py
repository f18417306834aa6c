"""ctypes binding of libnext_b200.so (the C ABI declared in include/next_gpu.h).

There is no fallback: if the CUDA library is missing or cannot be loaded,
:func:`load` raises.  Body arrays cross the boundary as float64 / int32 numpy
arrays in the caller's order.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("NEXT_B200_LIB") or os.path.join(HERE, "lib", "libnext_b200.so")

PHYSICS = {"reference": 0, "accurate": 1}
PRECISION = {"fp64": 0, "mixed": 1, "fp64group": 2}
DEVERR = {1: "tree capacity", 2: "walk stack", 4: "sort look-back timeout", 8: "interaction list"}


class Params(C.Structure):
    _fields_ = [("physics", C.c_int), ("precision", C.c_int), ("theta", C.c_double), ("eps", C.c_double),
                ("G", C.c_double), ("leaf_cap", C.c_int), ("group_cap", C.c_int), ("quadrupole", C.c_int),
                ("reuse_forces", C.c_int), ("walk_warps", C.c_int), ("walk_stack", C.c_int), ("device", C.c_int)]


class TuneResult(C.Structure):
    _fields_ = [("leaf_cap", C.c_int), ("group_cap", C.c_int), ("walk_warps", C.c_int), ("walk_stack", C.c_int),
                ("ms_force_phase", C.c_double), ("candidates", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("n_bodies", C.c_int64), ("n_systems", C.c_int64), ("n_nodes", C.c_int64),
                ("n_internal", C.c_int64), ("n_groups", C.c_int64), ("pp_interactions", C.c_int64),
                ("pc_interactions", C.c_int64), ("max_stack", C.c_int64), ("device_error", C.c_int32),
                ("steps", C.c_int32), ("ms_step", C.c_double), ("ms_build", C.c_double), ("ms_walk", C.c_double),
                ("ms_sort", C.c_double), ("ms_other", C.c_double), ("walk_launches", C.c_int64),
                ("key_levels", C.c_int32), ("recoveries", C.c_int32)]


# name -> (restype, argtypes)
_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int)
_i64 = C.POINTER(C.c_int64)
_u64 = C.POINTER(C.c_uint64)
_u32 = C.POINTER(C.c_uint32)
_h = C.c_void_p
SIGNATURES = {
    "next_params_default": (C.c_int, [C.POINTER(Params), C.c_int, C.c_int]),
    "next_create": (C.c_int, [C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "next_destroy": (None, [_h]),
    "next_last_error": (C.c_char_p, [_h]),
    "next_status_string": (C.c_char_p, [C.c_int]),
    "next_upload": (C.c_int, [_h, C.c_int64, _d, _d, _d, _d, _d, _d, _d, _i32]),
    "next_upload_systems": (C.c_int, [_h, C.c_int64, _i64, _d, _d, _d, _d, _d, _d, _d, _i32]),
    "next_download": (C.c_int, [_h, _d, _d, _d, _d, _d, _d]),
    "next_step": (C.c_int, [_h, C.c_double]),
    "next_steps": (C.c_int, [_h, C.c_double, C.c_int]),
    "next_step_host": (C.c_int, [_h, C.c_double, C.c_int64, _d, _d, _d, _d, _d, _d, _d, _i32]),
    "next_accel": (C.c_int, [_h, _d, _d, _d, _d]),
    "next_adaptive_dt": (C.c_int, [_h, C.c_double, _d]),
    "next_direct_accel": (C.c_int, [_h, C.c_int64, _i64, _d, _d, _d, _d]),
    "next_diagnostics": (C.c_int, [_h, _d]),
    "next_stats_get": (C.c_int, [_h, C.POINTER(Stats)]),
    "next_set_timing": (C.c_int, [_h, C.c_int]),
    "next_reset_timers": (C.c_int, [_h]),
    "next_sync": (C.c_int, [_h]),
    "next_debug_keys": (C.c_int, [_h, _u64, _d]),
    "next_debug_order": (C.c_int, [_h, _i64]),
    "next_debug_tree": (C.c_int, [_h, _d, C.c_int64, _i64]),
    "next_debug_fix_tree_capacity": (C.c_int, [_h, C.c_int64]),
    "next_debug_softening": (C.c_int, [C.c_int, C.c_int64, _d, _d, _d, _d]),
    "next_sort_pairs": (C.c_int, [_h, C.c_int64, _u64, _u32, _u64, _u32, C.c_int]),
    "next_fp32_peak": (C.c_int, [C.c_int, _d, _d]),
    "next_flush_l2": (C.c_int, [_h]),
    "next_autotune": (C.c_int, [_h, C.POINTER(TuneResult)]),
    "next_get_params": (C.c_int, [_h, C.POINTER(Params)]),
    "next_dist_unique_id": (C.c_int, [C.c_void_p]),
    "next_dist_attach": (C.c_int, [_h, C.c_int, C.c_int, C.c_void_p]),
    "next_host_alloc": (C.c_void_p, [C.c_int64]),
    "next_host_free": (None, [C.c_void_p]),
    "next_kernel_launches": (C.c_int64, []),
    "next_sort_pairs_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                          C.c_void_p]),
}

_LIB = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it is absent: there is no CPU path)."""
    global _LIB
    if _LIB is not None and path == LIB_PATH:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _LIB = lib
    return lib


class NextError(RuntimeError):
    pass


def dist_unique_id() -> bytes:
    """A fresh 128-byte NCCL unique id (made by rank 0 of a sharded run)."""
    lib = load()
    buf = C.create_string_buffer(128)
    rc = lib.next_dist_unique_id(buf)
    if rc:
        raise NextError(f"next_dist_unique_id failed ({rc})")
    return buf.raw


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def debug_softening(size, mass, dist, device: int = 0):
    """The device's reference softening law on arrays of (size, mass, dist)."""
    lib = load()
    size, mass, dist = _f64(size), _f64(mass), _f64(dist)
    out = np.empty(size.shape[0])
    rc = lib.next_debug_softening(device, size.shape[0], _p(size, _d), _p(mass, _d), _p(dist, _d), _p(out, _d))
    if rc:
        raise NextError(f"next_debug_softening failed ({rc})")
    return out


def fp32_peak(device: int = 0) -> float:
    lib = load()
    tf, mhz = C.c_double(0), C.c_double(0)
    rc = lib.next_fp32_peak(device, C.byref(tf), C.byref(mhz))
    if rc:
        raise NextError(f"next_fp32_peak failed ({rc})")
    return tf.value


class Simulation:
    """One device-resident N-body system (or a batch of independent systems)."""

    def __init__(self, physics: str = "accurate", precision: str = "mixed", **kw):
        self.lib = load()
        p = Params()
        rc = self.lib.next_params_default(C.byref(p), PHYSICS[physics], PRECISION[precision])
        if rc:
            raise NextError("next_params_default failed")
        for k, v in kw.items():
            if v is None:
                continue
            if k == "quadrupole":
                v = int(bool(v))
            if k == "reuse_forces":
                v = int(bool(v))
            setattr(p, k, v)
        self.params = p
        h = C.c_void_p()
        rc = self.lib.next_create(C.byref(p), C.byref(h))
        if rc:
            raise NextError(f"next_create failed: {self.lib.next_status_string(rc).decode()}")
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.next_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            msg = self.lib.next_last_error(self.h).decode()
            raise NextError(f"{what}: {self.lib.next_status_string(rc).decode()}: {msg}")

    def upload(self, b, offsets=None):
        n = int(b["x"].shape[0])
        arrs = [_f64(b[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        t = b.get("type")
        t = None if t is None else np.ascontiguousarray(t, dtype=np.int32)
        self._keep = (arrs, t)
        if offsets is None:
            rc = self.lib.next_upload(self.h, n, *(_p(a, _d) for a in arrs), _p(t, _i32))
        else:
            offs = np.ascontiguousarray(offsets, dtype=np.int64)
            rc = self.lib.next_upload_systems(self.h, offs.shape[0] - 1, _p(offs, _i64), *(_p(a, _d) for a in arrs),
                                              _p(t, _i32))
        self._check(rc, "upload")
        self.n = n

    def upload_arrays(self, arrs, t=None):
        """Upload from caller-owned float64 arrays (e.g. pinned host buffers) without copies."""
        rc = self.lib.next_upload(self.h, int(arrs[0].shape[0]), *(_p(a, _d) for a in arrs), _p(t, _i32))
        self._check(rc, "upload")
        self.n = int(arrs[0].shape[0])

    def download(self, out=None):
        n = self.n
        out = out if out is not None else {k: np.empty(n) for k in ("x", "y", "z", "vx", "vy", "vz")}
        rc = self.lib.next_download(self.h, *(_p(out.get(k), _d) for k in ("x", "y", "z", "vx", "vy", "vz")))
        self._check(rc, "download")
        return out

    def step(self, dt: float):
        self._check(self.lib.next_step(self.h, float(dt)), "step")

    def steps(self, dt: float, nsteps: int):
        self._check(self.lib.next_steps(self.h, float(dt), int(nsteps)), "steps")

    def step_host(self, lanes, dt: float, t=None):
        """One step on caller-owned float64 arrays, in place (the reference's Step()):
        lanes = [x, y, z, vx, vy, vz, m]; positions and velocities are overwritten."""
        n = int(lanes[0].shape[0])
        for a in lanes:
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape[0] != n:
                raise ValueError("step_host needs seven contiguous float64 arrays of one length")
        rc = self.lib.next_step_host(self.h, float(dt), n, *(_p(a, _d) for a in lanes), _p(t, _i32))
        self._check(rc, "step_host")
        self.n = n

    def accel(self, potential: bool = False):
        n = self.n
        a = {k: np.empty(n) for k in ("ax", "ay", "az")}
        pot = np.empty(n) if potential else None
        rc = self.lib.next_accel(self.h, _p(a["ax"], _d), _p(a["ay"], _d), _p(a["az"], _d), _p(pot, _d))
        self._check(rc, "accel")
        if potential:
            a["pot"] = pot
        return a

    def adaptive_dt(self, base_dt: float) -> float:
        out = C.c_double(0)
        self._check(self.lib.next_adaptive_dt(self.h, float(base_dt), C.byref(out)), "adaptive_dt")
        return out.value

    def direct_accel(self, idx):
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        k = idx.shape[0]
        a = {k2: np.empty(k) for k2 in ("ax", "ay", "az", "pot")}
        rc = self.lib.next_direct_accel(self.h, k, _p(idx, _i64), *(_p(a[c], _d) for c in ("ax", "ay", "az", "pot")))
        self._check(rc, "direct_accel")
        return a

    def diagnostics(self):
        out = np.zeros(8)
        self._check(self.lib.next_diagnostics(self.h, _p(out, _d)), "diagnostics")
        return {"kinetic": out[0], "potential": out[1], "momentum": out[2:5].copy(), "angular_momentum": out[5:8].copy()}

    def stats(self):
        s = Stats()
        self._check(self.lib.next_stats_get(self.h, C.byref(s)), "stats")
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def autotune(self):
        r = TuneResult()
        self._check(self.lib.next_autotune(self.h, C.byref(r)), "autotune")
        self.params = self.get_params()
        return {f: getattr(r, f) for f, _ in TuneResult._fields_}

    def get_params(self):
        p = Params()
        self._check(self.lib.next_get_params(self.h, C.byref(p)), "get_params")
        return p

    def dist_attach(self, rank: int, world: int, unique_id: bytes | None):
        """Join a sharded run (unique_id from dist_unique_id on rank 0); None: own share only."""
        buf = None if unique_id is None else C.create_string_buffer(bytes(unique_id), 128)
        self._check(self.lib.next_dist_attach(self.h, int(rank), int(world), buf), "dist_attach")

    def set_timing(self, on: bool):
        self._check(self.lib.next_set_timing(self.h, int(bool(on))), "set_timing")

    def reset_timers(self):
        self._check(self.lib.next_reset_timers(self.h), "reset_timers")

    def sync(self):
        self._check(self.lib.next_sync(self.h), "sync")

    def flush_l2(self):
        self._check(self.lib.next_flush_l2(self.h), "flush_l2")

    def debug_keys(self):
        keys = np.empty(self.n, dtype=np.uint64)
        cube = np.empty(4)
        self._check(self.lib.next_debug_keys(self.h, _p(keys, _u64), _p(cube, _d)), "debug_keys")
        return keys, cube

    def debug_order(self):
        perm = np.empty(self.n, dtype=np.int64)
        self._check(self.lib.next_debug_order(self.h, _p(perm, _i64)), "debug_order")
        return perm

    def debug_tree(self):
        cap = 4 * self.n + 64
        rows = np.zeros((cap, 16))
        nn = C.c_int64(0)
        self._check(self.lib.next_debug_tree(self.h, _p(rows, _d), cap, C.byref(nn)), "debug_tree")
        assert nn.value <= cap
        return rows[: nn.value]

    def debug_fix_tree_capacity(self, cap_internal: int):
        self._check(self.lib.next_debug_fix_tree_capacity(self.h, int(cap_internal)), "debug_fix_tree_capacity")

    def sort_pairs(self, keys, vals, key_bits: int = 64):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        vals = np.ascontiguousarray(vals, dtype=np.uint32)
        ko = np.empty_like(keys)
        vo = np.empty_like(vals)
        rc = self.lib.next_sort_pairs(self.h, keys.shape[0], _p(keys, _u64), _p(vals, _u32), _p(ko, _u64),
                                      _p(vo, _u32), int(key_bits))
        self._check(rc, "sort_pairs")
        return ko, vo
