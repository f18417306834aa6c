"""The CPU oracle against the golden fixtures produced by the reference.

Bit-exact: the oracle restates the reference's arithmetic in the same order
(oracle/bh_oracle.cpp is built with -ffp-contract=off, as the reference's
x86-64 build runs without FMA contraction).
"""
import numpy as np
import pytest

from golden_cases import NAMES, load, GOLDEN


@pytest.mark.parametrize("name", NAMES)
def test_tree_matches_reference(oracle, name):
    b, z = load(name)
    mine = oracle.tree(b, mode="ref")
    ref = z["tree"]
    assert mine.shape == ref.shape
    # level, mass, COM, half-width, quadrupole, leaf flag, body index
    np.testing.assert_array_equal(mine[:, :14], ref[:, :14])


@pytest.mark.parametrize("name", NAMES)
def test_keys_follow_reference_insertion_paths(oracle, name):
    b, z = load(name)
    keys = oracle.keys(b)
    depth = z["leaf_depth"]
    for k, path, d in zip(keys, z["leaf_paths"], depth):
        d = min(int(d), 21)
        mask = 0 if d == 0 else ((1 << 63) - (1 << (63 - 3 * d)))
        assert (int(k) & mask) == int(path)


@pytest.mark.parametrize("name", NAMES)
def test_accel_matches_reference(oracle, name):
    b, z = load(name)
    a = oracle.accel(b, mode="ref", theta=0.5)
    for c in ("ax", "ay", "az"):
        np.testing.assert_array_equal(a[c], z[c])


@pytest.mark.parametrize("name", NAMES)
def test_step_matches_reference(oracle, name):
    b, z = load(name)
    s = oracle.step(b, float(z["step_dt"]), int(z["nsteps"]), mode="ref")
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(s[c], z["out_" + c])


@pytest.mark.parametrize("name", NAMES)
def test_adaptive_dt_matches_reference(oracle, name):
    b, z = load(name)
    assert oracle.adaptive_dt(b, float(z["base_dt"])) == float(z["adaptive_dt"])


def test_sort_is_stable(oracle):
    keys = np.array([5, 3, 5, 1, 3, 3, 0, 5], dtype=np.uint64)
    perm = oracle.sort(keys)
    assert perm.tolist() == [6, 3, 1, 4, 5, 0, 2, 7]


def test_accurate_mode_against_direct_sum(oracle):
    from next_b200 import ic
    b = ic.plummer(4096, seed=0)
    idx = np.arange(0, 4096, 4)
    d = oracle.direct(b, idx, eps=0.01)
    for leaf_cap in (1, 8):
        a = oracle.accel(b, mode="accurate", theta=0.5, eps=0.01, leaf_cap=leaf_cap)
        num = np.sqrt(sum((a[c][idx] - d[c]) ** 2 for c in ("ax", "ay", "az")))
        den = np.sqrt(sum(d[c] ** 2 for c in ("ax", "ay", "az")))
        err = num / den
        assert np.median(err) < 1e-3
        assert np.percentile(err, 99) < 1e-2
