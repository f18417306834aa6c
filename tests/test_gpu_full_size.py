"""Full-size checks at the largest configured system (16,777,216 bodies).

At this size a CPU reference of the whole path would take hours, so these
tests check properties that do not depend on size: the key sort against
NumPy's stable sort, and for a Hernquist halo (theta = 0.7, eps = 0.002, the
16.7M workload) that KDK steps complete on the device, keep the momentum
within the force-error level, and leave forces within the accuracy target
against FP64 direct summation on sampled bodies.
"""
import numpy as np
import pytest

from next_b200 import ic
from next_b200.native import Simulation

N = 16_777_216

pytestmark = pytest.mark.gpu


def test_sort_at_full_size():
    rng = np.random.default_rng(44)
    keys = rng.integers(0, 2 ** 63, N, dtype=np.uint64)
    keys[::7] = keys[0]                      # duplicates: stability matters
    vals = np.arange(N, dtype=np.uint32)
    sim = Simulation("reference", "fp64")
    ko, vo = sim.sort_pairs(keys, vals, 63)
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(ko, keys[order])
    np.testing.assert_array_equal(vo, vals[order])
    sim.close()


def test_hernquist_halo_steps_on_device():
    b = ic.hernquist(N, seed=4)
    sim = Simulation("accurate", "mixed", theta=0.7, eps=0.002)
    sim.upload(b)
    p0 = sim.diagnostics()["momentum"]
    sim.steps(2.5e-4, 3)
    st = sim.stats()
    assert st["device_error"] == 0
    assert st["n_nodes"] > 0 and st["n_groups"] > N // 32
    state = sim.download()
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.all(np.isfinite(state[c]))
    p1 = sim.diagnostics()["momentum"]
    assert np.max(np.abs(p1 - p0)) < 1e-4
    a = sim.accel()                          # forces at the current positions
    idx = np.random.default_rng(5).choice(N, 1024, replace=False)
    d = sim.direct_accel(idx)                # FP64 direct summation on the device
    num = np.sqrt(sum((a[c][idx] - d[c]) ** 2 for c in ("ax", "ay", "az")))
    den = np.sqrt(sum(d[c] ** 2 for c in ("ax", "ay", "az")))
    err = num / den
    assert np.median(err) <= 1e-3
    assert np.percentile(err, 99) <= 1e-2
    sim.close()


def test_ballistic_drift_exact_above_inverse_split():
    """With G = 0 every body drifts ballistically: after two KDK steps of dt
    its position is (x + v dt) + v dt in FP64, which the host repeats
    exactly.  2,200,000 bodies is above the size from which the reorder
    leaves the inverse permutation (caller index -> position) to a launch of
    its own, so this checks that launch through every exported lane."""
    n = 2_200_000
    rng = np.random.default_rng(11)
    b = ic.uniform_sphere(n, seed=13)
    for c in ("vx", "vy", "vz"):
        b[c] = rng.normal(0.0, 0.1, n)
    sim = Simulation("accurate", "mixed", theta=0.5, eps=0.01, G=0.0)
    sim.upload(b)
    dt = 1e-3
    sim.steps(dt, 2)
    st = sim.download()
    for c, v in (("x", "vx"), ("y", "vy"), ("z", "vz")):
        expect = (b[c] + b[v] * dt) + b[v] * dt
        np.testing.assert_array_equal(st[c], expect)
        np.testing.assert_array_equal(st[v], b[v])
    assert sim.stats()["device_error"] == 0
    sim.close()
