"""Regenerate the golden fixtures in this folder from the reference itself.

The reference (NEXT) ships no tests, golden vectors or fixtures, so these
fixtures are produced by running the reference's own FP64 gravity code:
oracle/_ref/libnextref.so, which oracle/Makefile compiles from the
reference's unmodified headers (src/gravity/step.h, src/gravity/octree.h,
src/dt/softening.h, src/dt/adaptive.h).  Inputs are seeded synthetic bodies.

    make -C oracle && python tests/golden/make_golden.py

Each case is one .npz holding the inputs and the reference's outputs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from next_b200 import ic  # noqa: E402
from oracle.oracle import Reference  # noqa: E402


def _cases():
    rng = np.random.default_rng(1234)
    # 1. Plummer sphere with every 7th body a type-1 (dark matter) body, which
    #    exercises the reference's second softening rule (octree.h:146-148).
    b = ic.plummer(1024, seed=0)
    b["type"][::7] = 1
    yield "plummer1024_dm", b, dict(step_dt=1e-3, nsteps=3, base_dt=1e-2)
    # 2. Cold uniform sphere.
    yield "sphere512", ic.uniform_sphere(512, seed=1), dict(step_dt=5e-4, nsteps=4, base_dt=1e-3)
    # 3. Unequal masses, including zero-mass bodies (the walk skips m == 0 nodes).
    b = ic.plummer(300, seed=7)
    b["m"] = rng.uniform(0.0, 2.0, 300) / 300.0
    b["m"][::37] = 0.0
    yield "mixed_mass300", b, dict(step_dt=1e-3, nsteps=2, base_dt=1e-2)
    # 4. Bodies on a plane (zero z extent) and on a line (zero y and z extent).
    b = ic.plummer(200, seed=8)
    b["z"][:] = 0.0
    b["vz"][:] = 0.0
    yield "plane200", b, dict(step_dt=1e-3, nsteps=2, base_dt=1e-2)
    b = ic.plummer(64, seed=9)
    b["y"][:] = 0.25
    b["z"][:] = -0.5
    yield "line64", b, dict(step_dt=1e-3, nsteps=2, base_dt=1e-2)
    # 5. Tiny systems: one body, two bodies (the two-body example's masses),
    #    and the eight corners of a cube.
    one = {k: np.array([v]) for k, v in dict(x=0.3, y=-0.2, z=0.1, vx=0.0, vy=0.1, vz=0.0, m=1.0).items()}
    one["type"] = np.zeros(1, np.int32)
    yield "one_body", one, dict(step_dt=1e-3, nsteps=2, base_dt=1e-2)
    two = dict(x=np.array([0.0, 5.0]), y=np.zeros(2), z=np.zeros(2), vx=np.zeros(2),
               vy=np.array([0.0, 1.0]), vz=np.zeros(2), m=np.array([10.0, 1.0]),
               type=np.zeros(2, np.int32))
    yield "two_body", two, dict(step_dt=1e-3, nsteps=10, base_dt=1e-3)
    g = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=np.float64) * 2.0 - 1.0
    cube = dict(x=g[:, 0].copy(), y=g[:, 1].copy(), z=g[:, 2].copy(), vx=np.zeros(8), vy=np.zeros(8),
                vz=np.zeros(8), m=np.full(8, 0.125), type=np.zeros(8, np.int32))
    yield "cube8", cube, dict(step_dt=1e-2, nsteps=2, base_dt=1e-2)


def main():
    R = Reference()
    R.set_threads(1)
    for name, b, p in _cases():
        acc = R.accel(b)
        paths, depth = R.leaf_paths(b)
        tree = R.tree(b)
        st = R.step(b, p["step_dt"], p["nsteps"])
        dt = R.adaptive_dt(b, p["base_dt"])
        out = {f"in_{k}": np.asarray(b[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "type")}
        out.update({
            "ax": acc["ax"], "ay": acc["ay"], "az": acc["az"],
            "leaf_paths": paths, "leaf_depth": depth, "tree": tree,
            "step_dt": np.float64(p["step_dt"]), "nsteps": np.int64(p["nsteps"]),
            "base_dt": np.float64(p["base_dt"]), "adaptive_dt": np.float64(dt),
        })
        out.update({f"out_{k}": st[k] for k in ("x", "y", "z", "vx", "vy", "vz")})
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(f"{name}: n={b['x'].shape[0]} nodes={tree.shape[0]} max_depth={depth.max()}")
    # The reference softening law on a grid (src/dt/softening.h:21).
    sizes = np.geomspace(1e-5, 10.0, 13)
    masses = np.geomspace(1e-7, 1.0, 9)
    dists = np.concatenate([[0.0], np.geomspace(1e-6, 100.0, 11)])
    grid = np.array([[s, m, d, R.softening(s, m, d)] for s in sizes for m in masses for d in dists])
    np.savez_compressed(os.path.join(HERE, "softening_grid.npz"), grid=grid)
    print("softening_grid:", grid.shape[0], "points")


if __name__ == "__main__":
    main()
