"""Edge cases of the GPU path: systems of one and two bodies, ensembles that
hold empty and one-body systems, and a system far from the origin.

Tolerances
  * one body: zero force, and the drift x += v dt repeated exactly in FP64
  * two equal bodies: forces exactly opposite when they share a leaf (else
    within the magnitude tolerance); magnitude within 1e-14 (FP64) or 1e-6
    (FP32-mixed) of the softened two-body formula
  * ensembles: every non-empty system's forces bit-equal to that system
    uploaded alone (the existing ensemble rule)
  * offset system: mixed precision vs FP64 direct summation, median relative
    error <= 1e-3 and 99th percentile <= 1e-2 (FP32 terms are taken relative
    to each group's FP64 centre, so a large offset costs no accuracy)
"""
import numpy as np
import pytest

from next_b200 import ic
from next_b200.native import Simulation

pytestmark = pytest.mark.gpu


def bodies(pos, vel, mass):
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    vel = np.asarray(vel, dtype=np.float64).reshape(-1, 3)
    return {"x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy(),
            "vx": vel[:, 0].copy(), "vy": vel[:, 1].copy(), "vz": vel[:, 2].copy(),
            "m": np.asarray(mass, dtype=np.float64).copy()}


def rel_err(a, b):
    num = np.sqrt(sum((a[c] - b[c]) ** 2 for c in ("ax", "ay", "az")))
    den = np.sqrt(sum(b[c] ** 2 for c in ("ax", "ay", "az")))
    return num / np.where(den > 0, den, 1.0)


@pytest.mark.parametrize("physics,precision", [("reference", "fp64"), ("accurate", "fp64"), ("accurate", "mixed")])
def test_one_body_moves_ballistically(physics, precision):
    b = bodies([0.3, -0.2, 0.1], [1.0, 0.5, -0.25], [1.0])
    sim = Simulation(physics, precision)
    sim.upload(b)
    a = sim.accel()
    for c in ("ax", "ay", "az"):
        assert a[c][0] == 0.0
    dt = 1e-3
    for _ in range(4):
        sim.step(dt)
    sim.steps(dt, 3)
    s = sim.download()
    x = {k: b[k].copy() for k in ("x", "y", "z")}
    for _ in range(7):
        for k, v in (("x", "vx"), ("y", "vy"), ("z", "vz")):
            x[k] = x[k] + b[v] * dt
    for k, v in (("x", "vx"), ("y", "vy"), ("z", "vz")):
        np.testing.assert_array_equal(s[k], x[k])
        np.testing.assert_array_equal(s[v], b[v])
    assert sim.stats()["device_error"] == 0
    sim.close()


@pytest.mark.parametrize("precision,leaf_cap,tol", [("fp64", 1, 1e-14), ("fp64", 8, 1e-14), ("mixed", 16, 1e-6)])
def test_two_bodies_pull_equally_and_oppositely(precision, leaf_cap, tol):
    eps = 0.01
    b = bodies([[0.1, 0.2, -0.3], [-0.4, 0.05, 0.25]], np.zeros(6), [0.5, 0.5])
    sim = Simulation("accurate", precision, eps=eps, leaf_cap=leaf_cap)
    sim.upload(b)
    a = sim.accel()
    for c in ("ax", "ay", "az"):
        if leaf_cap >= 2:
            assert a[c][0] == -a[c][1]      # one leaf: the same body-body term, mirrored
        else:
            # one leaf each: either may be taken as a cell (its quadrupole is zero)
            assert abs(a[c][0] + a[c][1]) <= tol * abs(a[c][0])
    d = np.array([b["x"][1] - b["x"][0], b["y"][1] - b["y"][0], b["z"][1] - b["z"][0]])
    want = 0.5 * d / (d @ d + eps * eps) ** 1.5
    got = np.array([a["ax"][0], a["ay"][0], a["az"][0]])
    assert np.linalg.norm(got - want) <= tol * np.linalg.norm(want)
    sim.close()


def test_ensemble_with_empty_and_one_body_systems():
    sizes = [0, 1, 2, 3, 0, 700, 1, 2500, 0]
    parts = [ic.plummer(k, seed=40 + i) for i, k in enumerate(sizes) if k > 0]
    allb = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    for precision, leaf in (("fp64", 1), ("mixed", 16)):
        ens = Simulation("accurate", precision, leaf_cap=leaf)
        ens.upload(allb, offsets=offs)
        a = ens.accel()
        for s, k in enumerate(sizes):
            if k == 0:
                continue
            sl = slice(offs[s], offs[s + 1])
            one = Simulation("accurate", precision, leaf_cap=leaf)
            one.upload({c: v[sl] for c, v in allb.items()})
            a1 = one.accel()
            for c in ("ax", "ay", "az"):
                np.testing.assert_array_equal(a[c][sl], a1[c])
            one.close()
        ens.steps(1e-3, 3)
        st = ens.download()
        assert all(np.all(np.isfinite(st[c])) for c in st)
        assert ens.stats()["device_error"] == 0
        ens.close()


def test_far_offset_system_keeps_mixed_accuracy(oracle):
    n = 16_384
    b = ic.plummer(n, seed=7)
    shift = {"x": 1.0e4, "y": -3.0e3, "z": 5.0e2}
    far = {k: (v + shift[k] if k in shift else v.copy()) for k, v in b.items()}
    idx = np.random.default_rng(8).choice(n, 1024, replace=False)
    errs = []
    for case in (b, far):
        sim = Simulation("accurate", "mixed", theta=0.5, eps=0.01)
        sim.upload(case)
        a = sim.accel()
        d = oracle.direct(case, idx, eps=0.01)
        e = rel_err({c: a[c][idx] for c in a}, d)
        assert np.median(e) <= 1e-3
        assert np.percentile(e, 99) <= 1e-2
        assert sim.stats()["device_error"] == 0
        errs.append(np.median(e))
        sim.close()
    assert errs[1] <= 2.0 * errs[0]
