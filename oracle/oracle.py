"""ctypes front end for the CPU checkers (test infrastructure only).

``Oracle``    wraps liboracle.so, the CPU restatement in bh_oracle.cpp.
``Reference`` wraps _ref/libnextref.so, the reference's own gravity headers
              compiled by oracle/Makefile.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
use this module; the shipped library never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnextref.so")

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int)
_i64 = C.POINTER(C.c_int64)
_u64 = C.POINTER(C.c_uint64)


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32a(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        L.orc_root_cube.argtypes = [C.c_int64, _d, _d, _d, _d]
        L.orc_keys.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_int, _u64]
        L.orc_sort.argtypes = [C.c_int64, _u64, _i64]
        L.orc_accel.argtypes = [C.c_int64, _d, _d, _d, _d, _i32, C.c_int, C.c_double, C.c_double,
                                C.c_double, C.c_int, C.c_int, _d, _d, _d, _d, _i64]
        L.orc_direct.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_double, C.c_double, C.c_int64, _i64,
                                 _d, _d, _d, _d]
        L.orc_step.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _d, _d, _i32, C.c_int, C.c_double,
                               C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int]
        L.orc_adaptive_dt.argtypes = [C.c_int64, _d, _d, _d, C.c_double]
        L.orc_adaptive_dt.restype = C.c_double
        L.orc_tree_export.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_int, C.c_double, C.c_int, _d, C.c_int64]
        L.orc_tree_export.restype = C.c_int64

    def root_cube(self, b):
        x, y, z = _f64(b["x"]), _f64(b["y"]), _f64(b["z"])
        out = np.zeros(4)
        self.lib.orc_root_cube(x.shape[0], _p(x, _d), _p(y, _d), _p(z, _d), _p(out, _d))
        return out

    def keys(self, b, cube=None, levels=21):
        x, y, z = _f64(b["x"]), _f64(b["y"]), _f64(b["z"])
        cube = self.root_cube(b) if cube is None else _f64(cube)
        out = np.zeros(x.shape[0], dtype=np.uint64)
        self.lib.orc_keys(x.shape[0], _p(x, _d), _p(y, _d), _p(z, _d), _p(cube, _d), levels, _p(out, _u64))
        return out

    def sort(self, keys):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        perm = np.zeros(keys.shape[0], dtype=np.int64)
        self.lib.orc_sort(keys.shape[0], _p(keys, _u64), _p(perm, _i64))
        return perm

    def accel(self, b, mode="accurate", theta=0.5, eps=0.01, G=1.0, leaf_cap=1, quad=True,
              potential=False):
        n = b["x"].shape[0]
        x, y, z, m = (_f64(b[k]) for k in ("x", "y", "z", "m"))
        t = _i32a(b.get("type", np.zeros(n, np.int32)))
        ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
        pot = np.zeros(n) if potential else None
        counts = np.zeros(3, dtype=np.int64)
        self.lib.orc_accel(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(t, _i32),
                           0 if mode == "ref" else 1, theta, eps, G, leaf_cap, int(quad),
                           _p(ax, _d), _p(ay, _d), _p(az, _d), _p(pot, _d), _p(counts, _i64))
        out = {"ax": ax, "ay": ay, "az": az, "pp": int(counts[0]), "pc": int(counts[1]),
               "nodes": int(counts[2])}
        if potential:
            out["pot"] = pot
        return out

    def direct(self, b, idx, eps=0.01, G=1.0):
        n = b["x"].shape[0]
        x, y, z, m = (_f64(b[k]) for k in ("x", "y", "z", "m"))
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        k = idx.shape[0]
        ax, ay, az, pot = np.zeros(k), np.zeros(k), np.zeros(k), np.zeros(k)
        self.lib.orc_direct(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), eps, G, k, _p(idx, _i64),
                            _p(ax, _d), _p(ay, _d), _p(az, _d), _p(pot, _d))
        return {"ax": ax, "ay": ay, "az": az, "pot": pot}

    def step(self, b, dt, nsteps=1, mode="ref", theta=0.5, eps=0.01, G=1.0, leaf_cap=1, quad=True):
        s = {k: _f64(b[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        n = s["x"].shape[0]
        t = _i32a(b.get("type", np.zeros(n, np.int32)))
        self.lib.orc_step(n, *(_p(s[k], _d) for k in ("x", "y", "z", "vx", "vy", "vz", "m")),
                          _p(t, _i32), 0 if mode == "ref" else 1, theta, eps, G, leaf_cap, int(quad),
                          dt, nsteps)
        s["type"] = t
        return s

    def adaptive_dt(self, b, base_dt):
        vx, vy, vz = _f64(b["vx"]), _f64(b["vy"]), _f64(b["vz"])
        return self.lib.orc_adaptive_dt(vx.shape[0], _p(vx, _d), _p(vy, _d), _p(vz, _d), base_dt)

    def tree(self, b, mode="ref", theta=0.5, leaf_cap=1):
        n = b["x"].shape[0]
        x, y, z, m = (_f64(b[k]) for k in ("x", "y", "z", "m"))
        cap = 4 * n + 64
        rows = np.zeros((cap, 16))
        nn = self.lib.orc_tree_export(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d),
                                      0 if mode == "ref" else 1, theta, leaf_cap, _p(rows, _d), cap)
        assert nn <= cap
        return rows[:nn]


class Reference:
    """The reference's own FP64 gravity path (compiled from its headers)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference is present")
        L = self.lib = C.CDLL(path)
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_max_threads.restype = C.c_int
        L.ref_accel.argtypes = [C.c_int64, _d, _d, _d, _d, _i32, C.c_double, _d, _d, _d]
        L.ref_step.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _d, _d, _i32, C.c_double, C.c_int]
        L.ref_adaptive_dt.argtypes = [C.c_int64, _d, _d, _d, C.c_double]
        L.ref_adaptive_dt.restype = C.c_double
        L.ref_next_softening.argtypes = [C.c_double, C.c_double, C.c_double]
        L.ref_next_softening.restype = C.c_double
        L.ref_tree_export.argtypes = [C.c_int64, _d, _d, _d, _d, _d, C.c_int64]
        L.ref_tree_export.restype = C.c_int64
        L.ref_leaf_paths.argtypes = [C.c_int64, _d, _d, _d, _d, _u64, _i32]
        L.ref_accel_sample.argtypes = [C.c_int64, _d, _d, _d, _d, _i32, C.c_double, C.c_int64, _i64, _d, _d, _d]
        L.ref_save_snapshot.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _d, _d, _i32, C.c_int, C.c_char_p]

    def set_threads(self, k):
        self.lib.ref_set_threads(int(k))

    def max_threads(self):
        return self.lib.ref_max_threads()

    def accel(self, b, theta=0.5):
        n = b["x"].shape[0]
        x, y, z, m = (_f64(b[k]) for k in ("x", "y", "z", "m"))
        t = _i32a(b.get("type", np.zeros(n, np.int32)))
        ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.ref_accel(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(t, _i32), theta,
                           _p(ax, _d), _p(ay, _d), _p(az, _d))
        return {"ax": ax, "ay": ay, "az": az}

    def accel_sample(self, b, idx, theta=0.5):
        """bhAccel for the bodies idx only (one tree build, len(idx) walks)."""
        n = b["x"].shape[0]
        x, y, z, m = (_f64(b[k]) for k in ("x", "y", "z", "m"))
        t = _i32a(b.get("type", np.zeros(n, np.int32)))
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        k = idx.shape[0]
        ax, ay, az = np.zeros(k), np.zeros(k), np.zeros(k)
        self.lib.ref_accel_sample(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(t, _i32), theta, k,
                                  _p(idx, _i64), _p(ax, _d), _p(ay, _d), _p(az, _d))
        return {"ax": ax, "ay": ay, "az": az}

    def step(self, b, dt, nsteps=1):
        s = {k: _f64(b[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        n = s["x"].shape[0]
        t = _i32a(b.get("type", np.zeros(n, np.int32)))
        self.lib.ref_step(n, *(_p(s[k], _d) for k in ("x", "y", "z", "vx", "vy", "vz", "m")),
                          _p(t, _i32), dt, nsteps)
        s["type"] = t
        return s

    def adaptive_dt(self, b, base_dt):
        vx, vy, vz = _f64(b["vx"]), _f64(b["vy"]), _f64(b["vz"])
        return self.lib.ref_adaptive_dt(vx.shape[0], _p(vx, _d), _p(vy, _d), _p(vz, _d), base_dt)

    def softening(self, size, mass, dist):
        return self.lib.ref_next_softening(size, mass, dist)

    def tree(self, b):
        n = b["x"].shape[0]
        x, y, z, m = (_f64(b[k]) for k in ("x", "y", "z", "m"))
        cap = 4 * n + 64
        rows = np.zeros((cap, 16))
        nn = self.lib.ref_tree_export(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(rows, _d), cap)
        assert nn <= cap
        return rows[:nn]

    def save_snapshot(self, b, path, fmt):
        """Write `b` with the reference's SaveVTK (fmt "vtk") or SaveVTU (fmt "vtu")."""
        n = b["x"].shape[0]
        lanes = [_f64(b[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        t = _i32a(b.get("type", np.zeros(n, np.int32)))
        self.lib.ref_save_snapshot(n, *(_p(a, _d) for a in lanes), _p(t, _i32), int(fmt == "vtu"),
                                   str(path).encode())

    def leaf_paths(self, b):
        n = b["x"].shape[0]
        x, y, z, m = (_f64(b[k]) for k in ("x", "y", "z", "m"))
        paths = np.zeros(n, dtype=np.uint64)
        depth = np.zeros(n, dtype=np.int32)
        rc = self.lib.ref_leaf_paths(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d),
                                     _p(paths, _u64), _p(depth, _i32))
        if rc != 0:
            raise RuntimeError(f"ref_leaf_paths failed ({rc})")
        return paths, depth
