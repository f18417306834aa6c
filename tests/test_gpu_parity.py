"""GPU parity: the CUDA path against the oracle and the reference's own outputs.

Tolerances
  * octant keys, sort order, tree topology, reference-mode moments: bit-exact
  * reference physics, plain FP64 forces: relative 1e-10 per body against the
    compiled reference (same FP64 operations; only CUDA's cbrt/pow may differ
    from the host libm in the last bit), trajectories |x_gpu - x_ref| <=
    1e-12 * max|x_ref|
  * accurate physics, plain FP64 vs the oracle: 1e-12 relative
  * mixed precision vs FP64 direct summation: median relative error <= 1e-3
    (theta = 0.5, quadrupole), 99th percentile <= 1e-2
"""
import os

import numpy as np
import pytest

from golden_cases import NAMES, load
from next_b200 import ic
from next_b200.native import NextError, Simulation

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    num = np.sqrt(sum((a[c] - b[c]) ** 2 for c in ("ax", "ay", "az")))
    den = np.sqrt(sum(b[c] ** 2 for c in ("ax", "ay", "az")))
    return num / np.where(den > 0, den, 1.0)


def max_abs(a, b, keys):
    return max(float(np.max(np.abs(np.asarray(a[k]) - np.asarray(b[k])))) for k in keys)


def scale(a):
    return float(np.max(np.sqrt(a["ax"] ** 2 + a["ay"] ** 2 + a["az"] ** 2))) or 1.0


@pytest.fixture(scope="module")
def ref_sim():
    s = Simulation("reference", "fp64")
    yield s
    s.close()


# ---- keys and sort ----------------------------------------------------------

@pytest.mark.parametrize("name", NAMES)
def test_keys_bit_exact_golden(oracle, ref_sim, name):
    b, _ = load(name)
    ref_sim.upload(b)
    keys, cube = ref_sim.debug_keys()
    np.testing.assert_array_equal(cube, oracle.root_cube(b))
    np.testing.assert_array_equal(keys, oracle.keys(b))


@pytest.mark.parametrize("n", [100_003, 1_000_000])
def test_keys_bit_exact_large(oracle, ref_sim, n):
    b = ic.hernquist(n, seed=4) if n > 200_000 else ic.plummer(n, seed=11)
    ref_sim.upload(b)
    keys, _ = ref_sim.debug_keys()
    np.testing.assert_array_equal(keys, oracle.keys(b))


@pytest.mark.parametrize("n,bits", [(1, 64), (2, 64), (3839, 63), (3840, 63), (3841, 63), (100_000, 64),
                                    (1_000_003, 63), (65_536, 8), (200_000, 20)])
def test_sort_matches_stable_sort(ref_sim, n, bits):
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, 2 ** min(bits, 63), n, dtype=np.uint64)
    if bits == 64:
        keys = keys | (rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63))
    if n > 10:
        keys[: n // 3] = keys[0]           # many duplicates: stability matters
    vals = np.arange(n, dtype=np.uint32)
    ko, vo = ref_sim.sort_pairs(keys, vals, bits)
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(ko, keys[order])
    np.testing.assert_array_equal(vo, vals[order])


@pytest.mark.parametrize("n,bits", [(50_000, 12), (3841, 1), (200_000, 41)])
def test_sort_ignores_bits_above_key_bits(ref_sim, n, bits):
    # bits at and above key_bits take no part in the order (even those below
    # the next multiple of 8, which the last 8-bit pass would otherwise see)
    rng = np.random.default_rng(n * bits)
    keys = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    vals = rng.permutation(n).astype(np.uint32)
    ko, vo = ref_sim.sort_pairs(keys, vals, bits)
    order = np.argsort(keys & np.uint64((1 << bits) - 1), kind="stable")
    np.testing.assert_array_equal(ko, keys[order])
    np.testing.assert_array_equal(vo, vals[order])


def test_body_order_is_stable_key_order(oracle, ref_sim):
    b = ic.plummer(50_000, seed=3)
    ref_sim.upload(b)
    perm = ref_sim.debug_order()
    np.testing.assert_array_equal(perm, oracle.sort(oracle.keys(b)))


# ---- reference physics (plain FP64) against the reference -------------------

@pytest.mark.parametrize("name", NAMES)
def test_tree_matches_reference_golden(ref_sim, name):
    b, z = load(name)
    ref_sim.upload(b)
    mine = ref_sim.debug_tree()
    ref = z["tree"]
    assert mine.shape[0] == ref.shape[0]
    np.testing.assert_array_equal(mine[:, :14], ref[:, :14])


@pytest.mark.parametrize("name", NAMES)
def test_reference_forces_golden(ref_sim, name):
    b, z = load(name)
    ref_sim.upload(b)
    a = ref_sim.accel()
    ref = {c: z[c] for c in ("ax", "ay", "az")}
    assert max_abs(a, ref, ("ax", "ay", "az")) <= 1e-12 * scale(ref)


@pytest.mark.parametrize("name", NAMES)
def test_reference_step_golden(name):
    b, z = load(name)
    sim = Simulation("reference", "fp64")
    sim.upload(b)
    for _ in range(int(z["nsteps"])):
        sim.step(float(z["step_dt"]))
    s = sim.download()
    out = {c: z["out_" + c] for c in ("x", "y", "z", "vx", "vy", "vz")}
    tol = 1e-12 * max(1.0, max(float(np.max(np.abs(out[c]))) for c in out))
    assert max_abs(s, out, out.keys()) <= tol
    sim.close()


@pytest.mark.parametrize("name", NAMES)
def test_adaptive_dt_golden(ref_sim, name):
    b, z = load(name)
    ref_sim.upload(b)
    assert ref_sim.adaptive_dt(float(z["base_dt"])) == float(z["adaptive_dt"])


def test_reference_forces_plummer_64k(oracle, ref_sim):
    """Per body, relative 1e-10 against the compiled reference's own bhAccel
    (src/gravity/octree.h:133-179), with a fifth of the bodies of the dark-
    matter type (the second softening rule, octree.h:145-148); and against
    the CPU restatement on the same bodies."""
    from oracle.oracle import Reference
    b = ic.plummer(65_536, seed=0)
    b["type"][::5] = 1
    ref_sim.upload(b)
    a = ref_sim.accel()
    r = Reference().accel(b)
    e = rel_err(a, r)
    assert float(np.max(e)) <= 1e-10, float(np.max(e))
    o = oracle.accel(b, mode="ref")
    assert float(np.max(rel_err(a, o))) <= 1e-10


@pytest.mark.parametrize("name", NAMES)
def test_reference_forces_golden_per_body(ref_sim, name):
    """The golden cases body by body: relative 1e-10 wherever the reference's
    force is not zero, and exactly zero where it is."""
    b, z = load(name)
    ref_sim.upload(b)
    a = ref_sim.accel()
    ref = {c: z[c] for c in ("ax", "ay", "az")}
    mag = np.sqrt(ref["ax"] ** 2 + ref["ay"] ** 2 + ref["az"] ** 2)
    e = rel_err(a, ref)
    assert float(np.max(e[mag > 0], initial=0.0)) <= 1e-10
    for c in ("ax", "ay", "az"):
        assert not np.any(a[c][mag == 0])


def test_softening_law_on_the_golden_grid():
    """The device's nextSoftening (src/dt/softening.h:21-35) at every point of
    the grid the compiled reference was evaluated on (sizes 1e-5..10, masses
    1e-7..1, distances 0 and 1e-6..100): equal up to CUDA's cbrt rounding."""
    from next_b200.native import debug_softening
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "softening_grid.npz"))["grid"]
    got = debug_softening(g[:, 0], g[:, 1], g[:, 2])
    rel = np.abs(got - g[:, 3]) / g[:, 3]
    assert float(rel.max()) <= 1e-15, float(rel.max())
    # the 1e-4 floor is reproduced exactly
    floor = g[:, 3] == 1e-4
    assert floor.any() and np.all(got[floor] == 1e-4)


# ---- accurate physics --------------------------------------------------------

@pytest.mark.parametrize("leaf_cap", [1, 8])
def test_accurate_plain_matches_oracle(oracle, leaf_cap):
    b = ic.plummer(16_384, seed=2)
    sim = Simulation("accurate", "fp64", theta=0.5, eps=0.01, leaf_cap=leaf_cap)
    sim.upload(b)
    a = sim.accel(potential=True)
    r = oracle.accel(b, mode="accurate", theta=0.5, eps=0.01, leaf_cap=leaf_cap, potential=True)
    assert max_abs(a, r, ("ax", "ay", "az")) <= 1e-12 * scale(r)
    assert float(np.max(np.abs(a["pot"] - r["pot"]))) <= 1e-12 * float(np.max(np.abs(r["pot"])))
    st = sim.stats()
    assert st["pp_interactions"] == r["pp"] and st["pc_interactions"] == r["pc"]
    sim.close()


def test_direct_sum_matches_oracle(oracle):
    b = ic.plummer(20_000, seed=5)
    sim = Simulation("accurate", "mixed", eps=0.01)
    sim.upload(b)
    idx = np.arange(0, 20_000, 37)
    d = sim.direct_accel(idx)
    r = oracle.direct(b, idx, eps=0.01)
    assert max_abs(d, r, ("ax", "ay", "az")) <= 1e-12 * scale(r)
    sim.close()


@pytest.mark.parametrize("maker,n,theta,eps", [
    (ic.plummer, 16_384, 0.5, 0.01),
    (ic.uniform_sphere, 65_536, 0.5, 0.005),
    (ic.hernquist, 65_536, 0.7, 0.002),
])
def test_mixed_precision_force_error(oracle, maker, n, theta, eps):
    b = maker(n)
    sim = Simulation("accurate", "mixed", theta=theta, eps=eps)
    sim.upload(b)
    a = sim.accel()
    idx = np.random.default_rng(0).choice(n, 1024, replace=False)
    d = oracle.direct(b, idx, eps=eps)
    e = rel_err({c: a[c][idx] for c in a}, d)
    assert np.median(e) <= 1e-3
    assert np.percentile(e, 99) <= 1e-2
    assert sim.stats()["device_error"] == 0
    sim.close()


@pytest.mark.parametrize("maker,n,theta,eps", [
    (ic.plummer, 16_384, 0.5, 0.01),
    (ic.hernquist, 65_536, 0.7, 0.002),
])
def test_fp64_group_walk_is_the_mixed_walk_in_fp64(oracle, maker, n, theta, eps):
    """NEXT_PRECISION_FP64_GROUP walks exactly the interaction lists of the
    FP32-mixed walk (same PP and PC counts) in FP64: the two differ by FP32
    rounding only, and both meet the bar against FP64 direct summation."""
    b = maker(n)
    g = Simulation("accurate", "fp64group", theta=theta, eps=eps)
    x = Simulation("accurate", "mixed", theta=theta, eps=eps)
    g.upload(b)
    x.upload(b)
    ag, ax_ = g.accel(), x.accel()
    sg, sx = g.stats(), x.stats()
    assert sg["pp_interactions"] == sx["pp_interactions"] and sg["pc_interactions"] == sx["pc_interactions"]
    assert float(np.median(rel_err(ax_, ag))) <= 2e-6
    idx = np.random.default_rng(0).choice(n, 1024, replace=False)
    d = oracle.direct(b, idx, eps=eps)
    eg = rel_err({c: ag[c][idx] for c in ag}, d)
    assert np.median(eg) <= 1e-3 and np.percentile(eg, 99) <= 1e-2
    g.close()
    x.close()


def test_fp64_group_walk_opening_everything_is_direct_summation(oracle):
    """With theta -> 0 every cell is opened, so the FP64 group walk is a direct
    sum over all bodies in FP64: relative 1e-12 against the oracle, potential
    included."""
    b = ic.plummer(4096, seed=17)
    g = Simulation("accurate", "fp64group", theta=1e-4, eps=0.01)
    g.upload(b)
    a = g.accel(potential=True)
    d = oracle.direct(b, np.arange(4096), eps=0.01)
    assert float(np.max(rel_err(a, d))) <= 1e-12
    assert float(np.max(np.abs(a["pot"] - d["pot"]) / np.abs(d["pot"]))) <= 1e-12
    st = g.stats()
    assert st["pc_interactions"] == 0 and st["pp_interactions"] == 4096 * 4096
    g.close()


def test_fp64_group_graph_steps_equal_eager_steps():
    b = ic.plummer(20_000, seed=8)
    a = Simulation("accurate", "fp64group")
    g = Simulation("accurate", "fp64group")
    a.upload(b)
    g.upload(b)
    for _ in range(5):
        a.step(1e-3)
    g.steps(1e-3, 5)
    sa, sg = a.download(), g.download()
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(sa[c], sg[c])
    a.close()
    g.close()


def test_mixed_steps_trim_key_depth(oracle):
    """After the first build the FP32-mixed path keeps only the measured tree
    depth + 2 octant levels (or more, filling whole sort digits) in its keys;
    forces stay as accurate and match a
    full-depth build of the same state (same tree, bodies within a leaf may be
    in another order)."""
    b = ic.plummer(60_000, seed=21)
    sim = Simulation("accurate", "mixed", theta=0.5, eps=0.01)
    sim.upload(b)
    assert sim.stats()["key_levels"] == 21
    sim.steps(1e-3, 3)
    levels = sim.stats()["key_levels"]
    assert 3 < levels < 21
    a = sim.accel()
    state = sim.download()
    now = dict(b)
    now.update(state)
    full = Simulation("accurate", "mixed", theta=0.5, eps=0.01)
    full.upload(now)
    f = full.accel()
    assert full.stats()["key_levels"] == 21 or full.stats()["key_levels"] == levels
    assert np.median(rel_err(a, f)) <= 1e-5
    idx = np.random.default_rng(1).choice(60_000, 1024, replace=False)
    d = oracle.direct(now, idx, eps=0.01)
    assert np.median(rel_err({c: a[c][idx] for c in a}, d)) <= 1e-3
    assert sim.stats()["device_error"] == 0
    sim.close()
    full.close()


def test_key_depth_grows_with_the_tree():
    """Half the bodies fly ballistically (G = 0) into a small clump, so the
    tree deepens past the trimmed key depth.  The leaf over capacity this
    causes at the last key level is noticed at the next synchronisation and
    the keys get more levels; once they suffice, the tree matches a
    full-depth build of the same state."""
    n = 24_576
    b = ic.uniform_sphere(n, seed=7)
    target = {"x": 0.3, "y": 0.2, "z": 0.1}
    for ax in ("x", "y", "z"):
        v = np.zeros(n)
        v[n // 2:] = (target[ax] - b[ax][n // 2:]) / 0.95
        b["v" + ax] = v
    sim = Simulation("accurate", "mixed", theta=0.5, eps=0.001, G=0.0)
    sim.upload(b)
    sim.accel()
    start = sim.stats()["key_levels"]
    assert start < 21
    sim.steps(0.3, 3)
    for _ in range(8):
        before = sim.stats()["key_levels"]
        sim.reset_timers()
        sim.steps(0.0, 1)            # a step of zero length: a new build at the same positions
        if sim.stats()["key_levels"] == before:
            break
    st = sim.stats()
    assert st["key_levels"] > start
    now = dict(b)
    now.update(sim.download())
    full = Simulation("accurate", "mixed", theta=0.5, eps=0.001, G=0.0)
    full.upload(now)
    full.accel()
    full.reset_timers()
    full.steps(0.0, 1)
    fs = full.stats()
    keys = ("n_nodes", "n_internal", "n_groups")
    assert tuple(st[k] for k in keys) == tuple(fs[k] for k in keys)
    # groups may split a child at another body when bodies deeper than the
    # key levels keep their previous order: totals agree to a fraction
    mine = st["pp_interactions"] + st["pc_interactions"]
    ref = fs["pp_interactions"] + fs["pc_interactions"]
    assert abs(mine - ref) <= 0.01 * ref
    assert st["device_error"] == 0 and fs["device_error"] == 0
    sim.close()
    full.close()


def test_mixed_close_to_plain_accurate():
    b = ic.plummer(32_768, seed=6)
    plain = Simulation("accurate", "fp64", theta=0.5, eps=0.01, leaf_cap=16)
    mixed = Simulation("accurate", "mixed", theta=0.5, eps=0.01, leaf_cap=16)
    plain.upload(b)
    mixed.upload(b)
    e = rel_err(mixed.accel(), plain.accel())
    # different opening tests (group box vs body) -> truncation-level differences only
    assert np.median(e) <= 1e-3
    plain.close()
    mixed.close()


# ---- integration ---------------------------------------------------------------

def test_upload_download_round_trip():
    b = ic.plummer(10_000, seed=9)
    sim = Simulation("accurate", "mixed")
    sim.upload(b)
    s = sim.download()
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(s[c], b[c])
    sim.accel()           # reorders the bodies on the device
    s = sim.download()
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(s[c], b[c])
    sim.close()


def test_mixed_steps_conserve_energy_and_momentum():
    b = ic.plummer(32_768, seed=7)
    sim = Simulation("accurate", "mixed", theta=0.5, eps=0.01)
    sim.upload(b)
    d0 = sim.diagnostics()
    e0 = d0["kinetic"] + d0["potential"]
    sim.steps(1e-3, 50)
    d1 = sim.diagnostics()
    e1 = d1["kinetic"] + d1["potential"]
    assert abs(e1 - e0) / abs(e0) < 1e-4
    # Barnes-Hut forces are not pairwise symmetric: momentum drifts at the force-error level
    assert np.max(np.abs(d1["momentum"] - d0["momentum"])) < 2e-4
    assert sim.stats()["device_error"] == 0
    sim.close()


def test_graph_steps_equal_eager_steps():
    b = ic.plummer(20_000, seed=8)
    a = Simulation("accurate", "mixed")
    g = Simulation("accurate", "mixed")
    a.upload(b)
    g.upload(b)
    for _ in range(6):
        a.step(1e-3)
    g.steps(1e-3, 6)
    sa, sg = a.download(), g.download()
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(sa[c], sg[c])
    a.close()
    g.close()


def test_diagnostics_match_fp64_sums(oracle):
    """next_diagnostics against NumPy FP64 sums of the downloaded state:
    kinetic energy, momentum, angular momentum to 1e-12 relative; the
    potential energy (from the walk's potentials) against the FP64 direct
    sum over all bodies to the walk's accuracy."""
    b = ic.plummer(20_000, seed=19)
    b["m"] = b["m"] * np.random.default_rng(3).uniform(0.5, 1.5, 20_000)
    sim = Simulation("accurate", "mixed", eps=0.01)
    sim.upload(b)
    sim.steps(1e-3, 3)
    d = sim.diagnostics()
    s = sim.download()
    m = b["m"]
    T = 0.5 * np.sum(m * (s["vx"] ** 2 + s["vy"] ** 2 + s["vz"] ** 2))
    P = np.array([np.sum(m * s["vx"]), np.sum(m * s["vy"]), np.sum(m * s["vz"])])
    L = np.array([np.sum(m * (s["y"] * s["vz"] - s["z"] * s["vy"])),
                  np.sum(m * (s["z"] * s["vx"] - s["x"] * s["vz"])),
                  np.sum(m * (s["x"] * s["vy"] - s["y"] * s["vx"]))])
    assert abs(d["kinetic"] - T) <= 1e-12 * T
    pscale = np.sum(m * np.sqrt(s["vx"] ** 2 + s["vy"] ** 2 + s["vz"] ** 2))
    assert np.max(np.abs(d["momentum"] - P)) <= 1e-12 * pscale
    lscale = np.sum(m * np.sqrt(s["x"] ** 2 + s["y"] ** 2 + s["z"] ** 2)
                    * np.sqrt(s["vx"] ** 2 + s["vy"] ** 2 + s["vz"] ** 2))
    assert np.max(np.abs(d["angular_momentum"] - L)) <= 1e-12 * lscale
    now = dict(b)
    now.update(s)
    W = 0.5 * float(np.sum(m * oracle.direct(now, np.arange(20_000), eps=0.01)["pot"]))
    assert abs(d["potential"] - W) <= 1e-3 * abs(W)
    sim.close()


def test_graph_replay_recovers_from_tree_overflow():
    """A replayed step (next_steps) that overflows the tree capacity is finished
    the way next_step finishes it -- capacity grown, force phase and closing
    kick re-run -- and the replays after it, which did nothing, are taken
    again: the state equals the same steps taken one by one, bit for bit.

    The capacity is pinned (next_debug_fix_tree_capacity) to the largest
    internal-cell count of the replays before step j, where step j is the
    first whose tree needs more, so the overflow happens in a replay after
    the first, with replays queued behind it."""
    K, dt = 40, 5e-3
    for seed in range(8, 16):
        b = ic.plummer(20_000, seed=seed)
        ref = Simulation("accurate", "mixed")
        ref.upload(b)
        counts = [0]
        for _ in range(K):
            ref.step(dt)
            counts.append(ref.stats()["n_internal"])     # the build at the step's drifted positions
        # step 1 runs eagerly (it computes the first forces); steps 2..K replay
        j = next((j for j in range(3, K + 1) if counts[j] > max(counts[2:j])), None)
        if j is not None:
            break
        ref.close()
    assert j is not None, "no step needed a larger tree than step 2 for any seed"
    g = Simulation("accurate", "mixed")
    g.upload(b)
    g.step(dt)
    g.debug_fix_tree_capacity(max(counts[2:j]))
    g.steps(dt, K - 1)
    st = g.stats()
    assert st["recoveries"] == 1 and st["device_error"] == 0
    sr, sg = ref.download(), g.download()
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(sr[c], sg[c])
    # and the next call carries on from there
    ref.step(dt)
    g.steps(dt, 1)
    sr, sg = ref.download(), g.download()
    np.testing.assert_array_equal(sr["x"], sg["x"])
    ref.close()
    g.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_step_host_equals_upload_step_download(precision):
    """next_step_host (Step() on host arrays, positions copied back during the
    force phase, which with mixed precision replays a captured graph per buffer
    parity) gives the same state as next_upload + next_step + next_download.
    Four steps: both parities are captured and replayed."""
    b = ic.plummer(30_000, seed=12)
    s = Simulation("accurate", precision)
    h = Simulation("accurate", precision)
    names = ("x", "y", "z", "vx", "vy", "vz", "m")
    lanes = [np.ascontiguousarray(b[k], dtype=np.float64).copy() for k in names]
    ref = {k: np.ascontiguousarray(b[k], dtype=np.float64).copy() for k in names}
    for _ in range(4):
        s.upload_arrays([ref[k] for k in names])
        s.step(1e-3)
        s.download(ref)
        h.step_host(lanes, 1e-3)
        for i, k in enumerate(names[:6]):
            np.testing.assert_array_equal(lanes[i], ref[k])
    assert s.stats()["device_error"] == 0 and h.stats()["device_error"] == 0
    s.close()
    h.close()


def test_step_host_rejects_bad_input():
    b = ic.plummer(1_000, seed=13)
    h = Simulation("accurate", "mixed")
    names = ("x", "y", "z", "vx", "vy", "vz", "m")
    lanes = [np.ascontiguousarray(b[k], dtype=np.float64).copy() for k in names]
    keep = [a.copy() for a in lanes]
    lanes[0][5] = np.nan
    with pytest.raises(NextError):
        h.step_host(lanes, 1e-3)
    for a, k in zip(lanes[1:], keep[1:]):
        np.testing.assert_array_equal(a, k)      # nothing written back on failure
    lanes[0][5] = keep[0][5]
    with pytest.raises(NextError):
        h.step_host(lanes, float("inf"))
    h.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_step_host_with_changed_or_bad_inputs_between_calls(precision):
    """next_step_host starts each step on the state it returned last time
    while the new inputs upload, and keeps the result only if the inputs are
    that state bit for bit.  Unchanged inputs give what upload + step +
    download gives on a handle that holds the same state; inputs changed
    between calls (one velocity, one mass, one position by an ulp, a zero's
    sign) give the step of the changed state, equal to a new handle's upload +
    step + download of it; a call with bad inputs fails, writes nothing back
    and leaves the held state as the previous call returned it."""
    b = ic.plummer(20_000, seed=14)
    names = ("x", "y", "z", "vx", "vy", "vz", "m")
    lanes = [np.ascontiguousarray(b[k], dtype=np.float64).copy() for k in names]
    types = np.zeros(20_000, dtype=np.int32)
    h = Simulation("accurate", precision)
    ref = {}

    def fresh():
        # a new handle given the caller's current arrays
        f = Simulation("accurate", precision)
        for i, k in enumerate(names):
            ref[k] = lanes[i].copy()
        f.upload_arrays([ref[k] for k in names], types)
        return f

    def step_both(s):
        s.upload_arrays([ref[k] for k in names], types)
        s.step(1e-3)
        s.download(ref)
        h.step_host(lanes, 1e-3, types)
        for i, k in enumerate(names[:6]):
            np.testing.assert_array_equal(lanes[i], ref[k])

    s = fresh()
    step_both(s)
    step_both(s)                          # unchanged inputs: the speculative step is kept
    step_both(s)
    edits = [lambda: lanes[3].__setitem__(17, lanes[3][17] + 1e-3),
             lambda: lanes[6].__setitem__(400, lanes[6][400] * 1.5),
             lambda: lanes[2].__setitem__(1, np.nextafter(lanes[2][1], 1.0)),
             lambda: lanes[6].__setitem__(7, 0.0),
             lambda: lanes[6].__setitem__(7, -0.0)]          # the sign of a zero mass alone
    for edit in edits:
        edit()
        s.close()
        s = fresh()                       # the changed state, from scratch
        step_both(s)
        step_both(s)                      # and unchanged again afterwards
    # bad input on a speculative call: error, nothing written back
    keep = [a.copy() for a in lanes]
    lanes[6][3] = -1.0
    with pytest.raises(NextError):
        h.step_host(lanes, 1e-3, types)
    for a, k in zip(lanes[:6], keep[:6]):
        np.testing.assert_array_equal(a, k)
    lanes[6][3] = keep[6][3]
    s.close()
    s = fresh()                           # carries on from the state before the bad call
    step_both(s)
    step_both(s)
    assert s.stats()["device_error"] == 0 and h.stats()["device_error"] == 0
    s.close()
    h.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_one_rank_nccl_exchange_is_bit_identical(precision):
    """The sharded step's NCCL path on the one GPU a test gets: a one-rank
    communicator (ncclCommInitRank through the run-time loaded libnccl), the
    in-place all-gathers of every force phase -- eager and captured in the
    step graphs -- and the padded force lanes.  The state equals an
    unsharded handle's bit for bit."""
    from next_b200.native import dist_unique_id
    b = ic.plummer(20_000, seed=23)
    ref = Simulation("accurate", precision)
    one = Simulation("accurate", precision)
    ref.upload(b)
    one.upload(b)
    one.dist_attach(0, 1, dist_unique_id())
    for s_ in (ref, one):
        s_.step(1e-3)
        s_.steps(1e-3, 4)
    a, c = ref.accel(), one.accel()
    for k in ("ax", "ay", "az"):
        np.testing.assert_array_equal(a[k], c[k])
    sr, so = ref.download(), one.download()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(sr[k], so[k])
    assert one.stats()["device_error"] == 0
    ref.close()
    one.close()


def test_reuse_forces_matches_recompute():
    b = ic.plummer(20_000, seed=10)
    r = Simulation("accurate", "fp64", leaf_cap=4, reuse_forces=True)
    f = Simulation("accurate", "fp64", leaf_cap=4, reuse_forces=False)
    r.upload(b)
    f.upload(b)
    for _ in range(3):
        r.step(1e-3)
        f.step(1e-3)
    sr, sf = r.download(), f.download()
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(sr[c], sf[c])
    r.close()
    f.close()


def test_ensemble_equals_independent_systems():
    bodies, offs = ic.ensemble(n_systems=8, seed=3, nmin=500, nmax=5000)
    for precision, leaf in (("fp64", 1), ("mixed", 16), ("fp64group", 16)):
        ens = Simulation("accurate", precision, leaf_cap=leaf)
        ens.upload(bodies, offsets=offs)
        a = ens.accel()
        for s in range(8):
            sl = slice(offs[s], offs[s + 1])
            one = Simulation("accurate", precision, leaf_cap=leaf)
            one.upload({k: v[sl] for k, v in bodies.items()})
            b1 = one.accel()
            for c in ("ax", "ay", "az"):
                np.testing.assert_array_equal(a[c][sl], b1[c])
            one.close()
        ens.close()


def test_ensemble_steps_with_trimmed_keys_match_independent_systems():
    """Segmented keys with a trimmed key depth (system number right above the
    kept octant digits): stepping the batch matches stepping each system
    alone."""
    bodies, offs = ic.ensemble(n_systems=6, seed=5, nmin=2000, nmax=8000)
    ens = Simulation("accurate", "mixed")
    ens.upload(bodies, offsets=offs)
    ens.steps(1e-3, 3)
    assert ens.stats()["key_levels"] < 21
    got = ens.download()
    for s in range(6):
        sl = slice(offs[s], offs[s + 1])
        one = Simulation("accurate", "mixed")
        one.upload({k: v[sl] for k, v in bodies.items()})
        one.steps(1e-3, 3)
        want = one.download()
        # trees are the same; a group may still cut a leaf at another body
        # when the kept key levels differ, which moves forces by the
        # opening-test error (~1e-4 relative) on a few bodies
        for c in ("x", "y", "z"):
            np.testing.assert_allclose(got[c][sl], want[c], rtol=0, atol=1e-7)
        for c in ("vx", "vy", "vz"):
            np.testing.assert_allclose(got[c][sl], want[c], rtol=0, atol=1e-5)
        one.close()
    assert ens.stats()["device_error"] == 0
    ens.close()


def test_invalid_input_rejected():
    from next_b200.native import NextError
    b = ic.plummer(100, seed=1)
    b["x"][3] = np.nan
    sim = Simulation("accurate", "mixed")
    with pytest.raises(NextError):
        sim.upload(b)
    b = ic.plummer(100, seed=1)
    b["m"][5] = -1.0
    with pytest.raises(NextError):
        sim.upload(b)
    with pytest.raises(NextError):
        sim.step(1e-3)       # nothing uploaded
    sim.close()


def test_coincident_bodies_do_not_break_the_build():
    # the reference recurses forever on duplicates (octree.h:69-87); here they
    # share a deepest-level leaf
    b = ic.plummer(4096, seed=12)
    for k in ("x", "y", "z"):
        b[k][100:164] = b[k][99]
    for physics, precision in (("reference", "fp64"), ("accurate", "fp64"), ("accurate", "mixed")):
        sim = Simulation(physics, precision)
        sim.upload(b)
        a = sim.accel()
        assert all(np.all(np.isfinite(a[c])) for c in a)
        assert sim.stats()["device_error"] == 0
        sim.close()


def test_autotune_keeps_accuracy_and_state(oracle):
    b = ic.uniform_sphere(65_536, seed=21)
    sim = Simulation("accurate", "mixed", theta=0.5, eps=0.005)
    sim.upload(b)
    r = sim.autotune()
    assert r["candidates"] >= 12 and r["leaf_cap"] <= r["group_cap"] <= 32
    p = sim.get_params()
    assert (p.leaf_cap, p.group_cap, p.walk_warps) == (r["leaf_cap"], r["group_cap"], r["walk_warps"])
    s = sim.download()                       # tuning does not move bodies
    for c in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(s[c], b[c])
    a = sim.accel()
    idx = np.arange(0, 65_536, 64)
    e = rel_err({c: a[c][idx] for c in a}, oracle.direct(b, idx, eps=0.005))
    assert np.median(e) <= 1e-3
    sim.step(5e-4)
    assert sim.stats()["device_error"] == 0
    sim.close()


@pytest.mark.parametrize("precision,world", [("mixed", 2), ("mixed", 3), ("fp64", 2)])
def test_sharded_shares_equal_single_device(precision, world):
    """Each rank walks only its share of the bodies (key order); stitched, the
    shares equal the one-device forces bit for bit.  Ranks are emulated on one
    device (no communicator: next_dist_attach with id NULL)."""
    from next_b200.dist import partition
    b = ic.plummer(50_000, seed=31)
    leaf = 16 if precision == "mixed" else 1
    full = Simulation("accurate", precision, leaf_cap=leaf)
    full.upload(b)
    want = full.accel()
    order = full.debug_order()
    got = {c: np.full(50_000, np.nan) for c in ("ax", "ay", "az")}
    total_pc = 0
    for r in range(world):
        s = Simulation("accurate", precision, leaf_cap=leaf)
        s.upload(b)
        s.dist_attach(r, world, None)
        a = s.accel()
        np.testing.assert_array_equal(s.debug_order(), order)     # identical trees on every rank
        lo, hi, _ = partition(50_000, world, r)
        mine = order[lo:hi]
        for c in got:
            got[c][mine] = a[c][mine]
        total_pc += s.stats()["pc_interactions"]
        s.close()
    for c in got:
        np.testing.assert_array_equal(got[c], want[c])
    assert total_pc == full.stats()["pc_interactions"]
    full.close()


def test_timed_graph_replays_report_stages():
    b = ic.plummer(40_000, seed=41)
    sim = Simulation("accurate", "mixed")
    sim.upload(b)
    sim.step(1e-3)
    sim.reset_timers()
    sim.set_timing(True)
    sim.steps(1e-3, 5)
    sim.set_timing(False)
    st = sim.stats()
    assert st["steps"] == 5 and st["walk_launches"] == 5
    assert st["ms_walk"] > 0 and st["ms_build"] > 0 and st["ms_sort"] > 0
    assert st["ms_step"] >= st["ms_walk"] + st["ms_build"] - 1e-3
    assert st["pc_interactions"] > 0 and st["device_error"] == 0
    sim.close()
