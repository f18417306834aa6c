"""Benchmark: particle-steps/s of the KDK Barnes-Hut step on one B200.

Workload (default): cold collapse, N = 1,048,576 equal-mass bodies uniform in
the unit sphere, zero velocities, G = 1, eps = 0.005, theta = 0.5,
quadrupole, dt = 5e-4, seed 1.  A step is one full KDK step of the whole
system (tree build + force walk + kick/drift), bodies resident on the device.

The JSON line's `value` is the FP32-mixed step (FP32 interactions with
compensated accumulation, FP64 kick/drift, moments and diagnostics).  Beside
it: the plain FP64 GPU step (one thread per body, the reference's step
structure: two tree builds per step), the force error of both against FP64
direct summation on 4096 seeded bodies, the walk's FP32-pipe roofline, the
reference's own OpenMP Step() timed on the host cores, and an end-to-end
figure through the C ABI with host buffers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at <=1e-3 median force err: FP32-mixed vs FP64 GPU vs CPU"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FLOPS_PP, FLOPS_PC = 20, 56
# DRAM bytes (read + write) of one walk launch on this workload, from an ncu
# capture of the same command (dram__bytes_read.sum + dram__bytes_write.sum).
WALK_DRAM_BYTES = 56.32e6
L2_BYTES = 126 * 2 ** 20


def sort_passes(key_levels, n_systems):
    """Onesweep passes of the key sort: ceil(key_bits / 8), key_bits = the
    octant digits kept (3 per level; all 63 bits below the system number at
    full depth) plus the bits of the system number."""
    sys_bits = 0 if n_systems <= 1 else int(math.ceil(math.log2(n_systems)))
    full = min(21, (63 - sys_bits) // 3)
    base = 63 - sys_bits if key_levels >= full else 3 * key_levels
    return -(-(base + sys_bits) // 8)


def sort_bytes_per_body(passes):
    # each pass reads and writes a (u64 key, u32 index) pair; the histogram pass reads the keys once
    return passes * 24 + 8


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class Clocks:
    """nvidia-smi sampler for the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1])]
        mx = [num(r[2]) for r in rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        busy = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((num(r[3]) or 0.0) for r in rows)}


def measured_peaks():
    try:
        return json.load(open(PEAKS_FILE))
    except (OSError, ValueError):
        return {}


def force_error(a, d, idx):
    num = np.sqrt(sum((a[c][idx] - d[c]) ** 2 for c in ("ax", "ay", "az")))
    den = np.sqrt(sum(d[c] ** 2 for c in ("ax", "ay", "az")))
    e = num / den
    return {"median": float(np.median(e)), "p90": float(np.percentile(e, 90)), "p99": float(np.percentile(e, 99))}


def time_cpu_reference(bodies, dt, budget_s, threads=None):
    """The reference's own Step() (oracle/_ref, OpenMP on the host cores) on the same bodies."""
    from oracle.oracle import Reference
    R = Reference()
    threads = threads or os.cpu_count() or 1
    R.set_threads(threads)
    n = bodies["x"].shape[0]
    steps, t_total = 0, 0.0
    b = dict(bodies)
    while steps < 1 or (t_total < budget_s and steps < 50):
        t0 = time.perf_counter()
        b = R.step(b, dt, 1)
        t_total += time.perf_counter() - t0
        steps += 1
    return {"value": n * steps / t_total, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
            "sample": f"{steps} Step() call(s) of the reference (src/gravity/step.h) on the full "
                      f"{n}-body system, OpenMP {threads} threads, {t_total:.1f} s"}


def run_reference_arm(args):
    WORKLOAD = CONFIGS["c2"]
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from next_b200 import ic
    bodies = ic.uniform_sphere(WORKLOAD["n"], seed=WORKLOAD["seed"])
    steps = max(1, min(args.steps, 2))
    from oracle.oracle import Reference
    R = Reference()
    threads = os.cpu_count() or 1
    R.set_threads(threads)
    b = dict(bodies)
    warm = min(args.warmup, 3)
    for _ in range(warm):
        b = R.step(b, WORKLOAD["dt"], 1)
    t0 = time.perf_counter()
    for _ in range(steps):
        b = R.step(b, WORKLOAD["dt"], 1)
    t = time.perf_counter() - t0
    value = WORKLOAD["n"] * steps / t
    # the reference's as-shipped forces on 4096 seeded bodies of the initial
    # state against FP64 direct summation (CPU oracle) with the workload's eps
    from oracle.oracle import Oracle
    idx = np.random.default_rng(12345).choice(WORKLOAD["n"], 4096, replace=False)
    a = R.accel_sample(bodies, idx)
    d = Oracle().direct(bodies, idx, eps=WORKLOAD["eps"])
    ferr = force_error(a, d, np.arange(idx.shape[0]))
    ferr["versus"] = (f"FP64 direct summation with Plummer eps {WORKLOAD['eps']} on 4096 sampled bodies of the "
                      f"initial state (the reference's own softening differs)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * t / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD["name"], "n_bodies": WORKLOAD["n"], "theta": WORKLOAD["theta"],
                   "eps": "adaptive (reference softening law)", "dt": WORKLOAD["dt"], "seed": WORKLOAD["seed"],
                   "physics": "reference as shipped", "l2": "host run"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                         "sample": f"{steps} timed Step() call(s) on the full system after "
                                   f"{warm} warm-up; bounded so the run ends in minutes",
                         "force_error": ferr},
        "force_error": ferr,
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


CONFIGS = {
    "c1": dict(name="plummer_16k", maker="plummer", n=16_384, seed=0, eps=0.01, theta=0.5, dt=1e-3, steps=100),
    "c2": dict(name="cold_collapse_uniform_sphere", maker="uniform_sphere", n=1_048_576, seed=1, eps=0.005,
               theta=0.5, dt=5e-4, steps=200),
    "c3": dict(name="two_galaxy_encounter", maker="two_galaxies", n=4_194_304, seed=2, eps=0.01, theta=0.6, dt=1e-3,
               steps=100),
    "c4": dict(name="batched_plummer_ensemble_256", maker="ensemble", n=None, seed=3, eps=0.01, theta=0.5, dt=1e-3,
               steps=100),
    "c5": dict(name="hernquist_halo_16M", maker="hernquist", n=16_777_216, seed=4, eps=0.002, theta=0.7, dt=2.5e-4,
               steps=50),
}


def full_run(args):
    """The workload's whole configured run (its step count and dt) from the
    initial bodies through next_steps -- one graph replay per step, device
    error word checked every 64 replays with overflow recovery -- reporting
    completion, device time and the FP64 energy / momentum drift."""
    from next_b200.native import Simulation
    W = dict(CONFIGS[args.config])
    bodies, offsets = make_bodies(W)
    n = bodies["x"].shape[0]
    precision = args.precision
    sim = Simulation("accurate", precision, theta=W["theta"], eps=W["eps"])
    sim.upload(bodies, offsets=offsets)
    tune = sim.autotune()                        # positions unchanged
    d0 = sim.diagnostics()
    m = bodies["m"]
    pscale = float(np.sum(m * np.sqrt(bodies["vx"] ** 2 + bodies["vy"] ** 2 + bodies["vz"] ** 2)))
    sim.sync()
    sim.reset_timers()
    sim.set_timing(True)
    t0 = time.perf_counter()
    sim.steps(W["dt"], W["steps"])
    sim.sync()
    wall = time.perf_counter() - t0
    sim.set_timing(False)
    st = sim.stats()
    d1 = sim.diagnostics()
    e0, e1 = d0["kinetic"] + d0["potential"], d1["kinetic"] + d1["potential"]
    final = {k: v for k, v in sim.download().items()}
    vmag = np.sqrt(final["vx"] ** 2 + final["vy"] ** 2 + final["vz"] ** 2)
    pscale = max(pscale, float(np.sum(m * vmag)))
    err = None
    if offsets is None:
        idx = np.random.default_rng(12345).choice(n, min(4096, n), replace=False)
        err = force_error(sim.accel(), sim.direct_accel(idx), idx)
    sim.close()
    line = {"full_run": W["name"], "precision": precision, "n_bodies": n, "steps": W["steps"], "dt": W["dt"],
            "completed": st["steps"] == W["steps"] and st["device_error"] == 0,
            "device_ms": st["ms_step"], "ms_per_step": st["ms_step"] / max(1, st["steps"]), "wall_s": wall,
            "particle_steps_per_s": n * W["steps"] / (st["ms_step"] * 1e-3),
            "energy": {"E0": e0, "E1": e1, "rel_drift": abs(e1 - e0) / abs(e0), "T1_over_W1": d1["kinetic"] / abs(d1["potential"])},
            "momentum_drift": float(np.linalg.norm(d1["momentum"] - d0["momentum"])) / pscale,
            "recoveries": st["recoveries"], "key_levels": st["key_levels"], "force_error_end": err,
            "autotune": tune}
    print(json.dumps(line), flush=True)
    return 0


def make_bodies(cfg):
    from next_b200 import ic
    m = cfg["maker"]
    if m == "uniform_sphere":
        return ic.uniform_sphere(cfg["n"], seed=cfg["seed"]), None
    if m == "plummer":
        return ic.plummer(cfg["n"], seed=cfg["seed"]), None
    if m == "hernquist":
        return ic.hernquist(cfg["n"], seed=cfg["seed"]), None
    if m == "two_galaxies":
        return ic.two_galaxies(cfg["n"] // 2, seed=cfg["seed"]), None
    return ic.ensemble(256, seed=cfg["seed"])


def ensemble_error(bodies, offsets, a, cfg, device, k_systems=8):
    """Force error of the batched walk on a sample of systems, each against its own FP64 direct sum."""
    from next_b200.native import Simulation
    rng = np.random.default_rng(777)
    pick = rng.choice(len(offsets) - 1, k_systems, replace=False)
    errs = []
    for s in pick:
        sl = slice(offsets[s], offsets[s + 1])
        one = Simulation("accurate", "fp64", theta=cfg["theta"], eps=cfg["eps"], device=device)
        one.upload({k: v[sl] for k, v in bodies.items()})
        idx = np.arange(offsets[s + 1] - offsets[s])
        d = one.direct_accel(idx)
        num = np.sqrt(sum((a[c][sl] - d[c]) ** 2 for c in ("ax", "ay", "az")))
        den = np.sqrt(sum(d[c] ** 2 for c in ("ax", "ay", "az")))
        errs.append(num / den)
        one.close()
    e = np.concatenate(errs)
    return {"median": float(np.median(e)), "p90": float(np.percentile(e, 90)), "p99": float(np.percentile(e, 99)),
            "systems": int(k_systems)}


def plain_fp64_leg(bodies, offsets, cfg, device, steps, idx):
    """The plain FP64 GPU step (one thread per body, two tree builds per step)."""
    from next_b200.native import Simulation
    if offsets is None:
        p = Simulation("accurate", "fp64", theta=cfg["theta"], eps=cfg["eps"], leaf_cap=1, reuse_forces=False,
                       device=device)
        p.upload(bodies)
        p.step(cfg["dt"])
        p.sync()
        a_plain = p.accel()
        err = force_error(a_plain, p.direct_accel(idx), idx)
        p.reset_timers()
        p.set_timing(True)
        for _ in range(steps):
            p.flush_l2()
            p.step(cfg["dt"])
        p.sync()
        st = p.stats()
        p.close()
        n = bodies["x"].shape[0]
        return {"value": n * steps / (st["ms_step"] * 1e-3), "steps": steps, "ms_per_step": st["ms_step"] / steps,
                "force_error": err, "structure": "one thread per body, leaf_cap 1, two tree builds per step"}
    # ensemble: loop the single-system plain FP64 step over a sample of systems
    rng = np.random.default_rng(99)
    pick = rng.choice(len(offsets) - 1, 16, replace=False)
    bodies_done, ms = 0, 0.0
    for s in pick:
        sl = slice(offsets[s], offsets[s + 1])
        p = Simulation("accurate", "fp64", theta=cfg["theta"], eps=cfg["eps"], leaf_cap=1, reuse_forces=False,
                       device=device)
        p.upload({k: v[sl] for k, v in bodies.items()})
        p.step(cfg["dt"])
        p.reset_timers()
        p.set_timing(True)
        for _ in range(steps):
            p.step(cfg["dt"])
        p.sync()
        ms += p.stats()["ms_step"]
        bodies_done += (offsets[s + 1] - offsets[s]) * steps
        p.close()
    return {"value": bodies_done / (ms * 1e-3), "steps": steps, "ms_per_step": None, "force_error": None,
            "structure": "single-system plain FP64 step looped over 16 sampled systems (device time summed)"}


def fp64_group_leg(bodies, offsets, cfg, device, steps, idx, d_direct, prm):
    """The same algorithm in FP64: the group walk with the mixed run's tuned
    leaf, group and block settings (so the same tree, groups and interaction
    lists), force reuse and one graph replay per step -- only the precision of
    the interactions differs from the headline step."""
    from next_b200.native import Simulation
    g = Simulation("accurate", "fp64group", theta=cfg["theta"], eps=cfg["eps"], device=device,
                   leaf_cap=prm.leaf_cap, group_cap=prm.group_cap, walk_warps=prm.walk_warps,
                   walk_stack=prm.walk_stack)
    g.upload(bodies, offsets=offsets)
    err = force_error(g.accel(), d_direct, idx) if d_direct is not None else None
    g.steps(cfg["dt"], 2)
    g.sync()
    g.reset_timers()
    g.set_timing(True)
    for _ in range(steps):
        g.flush_l2()
        g.steps(cfg["dt"], 1)
    g.sync()
    st = g.stats()
    g.close()
    n = bodies["x"].shape[0]
    flops = (FLOPS_PP * st["pp_interactions"] + FLOPS_PC * st["pc_interactions"]) / max(1, st["walk_launches"])
    return {"value": n * steps / (st["ms_step"] * 1e-3), "unit": "particle-steps/s", "steps": steps,
            "ms_per_step": st["ms_step"] / steps, "walk_ms": st["ms_walk"] / max(1, st["walk_launches"]),
            "walk_tflops": flops / (st["ms_walk"] / max(1, st["walk_launches"]) * 1e-3) / 1e12,
            "force_error": err,
            "structure": "FP64 group walk: the mixed step's tree, groups, lists, force reuse and graph replay"}


def ref_physics_leg(bodies, cfg, device, steps, idx, d_direct, cpu_accel):
    """The drop-in default: reference physics (adaptive softening, the
    reference's opening test and quadrupole) in plain FP64 on the GPU -- what
    Step() and the `next` CLI run -- timed over `steps` KDK steps."""
    from next_b200.native import Simulation
    p = Simulation("reference", "fp64", device=device)
    p.upload(bodies)
    a = p.accel()
    err = force_error(a, d_direct, idx) if d_direct is not None else None
    parity = None
    if cpu_accel is not None:
        num = np.sqrt(sum((a[c][idx] - cpu_accel[c]) ** 2 for c in ("ax", "ay", "az")))
        den = np.sqrt(sum(cpu_accel[c] ** 2 for c in ("ax", "ay", "az")))
        parity = float(np.max(num / den))
    p.step(cfg["dt"])
    p.sync()
    p.reset_timers()
    p.set_timing(True)
    for _ in range(steps):
        p.flush_l2()
        p.step(cfg["dt"])
    p.sync()
    st = p.stats()
    p.close()
    n = bodies["x"].shape[0]
    return {"value": n * steps / (st["ms_step"] * 1e-3), "unit": "particle-steps/s", "steps": steps,
            "ms_per_step": st["ms_step"] / steps, "force_error": err,
            "max_rel_diff_vs_reference_cpu": parity,
            "physics": "reference (as the CPU arm: adaptive softening, half-width theta 0.5, its quadrupole)",
            "structure": "one thread per body, one body per leaf, two tree builds per step (step.h:113,164)"}


def large_sort_leg(cfg, device, n=8_388_608, steps=3):
    """The key sort at a size whose ping-pong buffers exceed the 126 MB L2:
    the same workload at n bodies, sort stage of `steps` eager steps."""
    from next_b200 import ic
    from next_b200.native import Simulation
    b = ic.uniform_sphere(n, seed=cfg["seed"])
    sim = Simulation("accurate", "mixed", theta=cfg["theta"], eps=cfg["eps"], device=device)
    sim.upload(b)
    sim.steps(cfg["dt"], 2)
    sim.sync()
    sim.reset_timers()
    sim.set_timing(True)
    for _ in range(steps):
        sim.flush_l2()
        sim.step(cfg["dt"])
    sim.sync()
    st = sim.stats()
    sim.close()
    passes = sort_passes(st["key_levels"], 1)
    ms = st["ms_sort"] / steps
    gbs = sort_bytes_per_body(passes) * n / (ms * 1e-3) / 1e9
    peak = measured_peaks().get("hbm_gbs")
    return {"n_bodies": n, "passes": passes, "bytes_per_body": sort_bytes_per_body(passes), "ms": ms,
            "gbs": gbs, "frac": gbs / peak if peak else None,
            "note": "ping-pong buffers of 24 B/body x 2 exceed the L2: an HBM figure"}


def run_ours(args):
    rank, world, local = env_rank()
    from next_b200.native import Simulation, fp32_peak, load
    lib = load()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                 timeout=__import__("datetime").timedelta(seconds=120))
        dist = tdist
    W = dict(CONFIGS[args.config])
    if args.n:
        W["n"] = args.n
        W["name"] = f"{W['name']}_n{args.n}"
    bodies, offsets = make_bodies(W)
    sharded = world > 1 and offsets is None      # one system over all ranks (force all-gather)
    if world > 1 and offsets is not None:
        # independent systems: each rank integrates whole systems, balanced by
        # N log N work (the same split on every rank), no collective
        from next_b200.dist import select_systems, split_systems
        mine = split_systems(np.diff(offsets), world)[rank]
        bodies, offsets = select_systems(bodies, offsets, mine)
    n = bodies["x"].shape[0]
    knobs = dict(leaf_cap=args.leaf_cap, group_cap=args.group_cap, walk_warps=args.walk_warps,
                 walk_stack=args.walk_stack)
    sim = Simulation("accurate", "mixed", theta=W["theta"], eps=W["eps"], device=local, **knobs)
    sim.upload(bodies, offsets=offsets)
    sim.step(W["dt"])
    tune = None if args.no_autotune else sim.autotune()
    if sharded:
        # every rank must build the same tree: rank 0's tuned setting goes to all,
        # and all ranks restart from the same initial bodies
        from next_b200.dist import attach
        import torch
        p = sim.get_params()
        t = torch.tensor([p.leaf_cap, p.group_cap, p.walk_warps, p.walk_stack], device=f"cuda:{local}")
        dist.broadcast(t, src=0)
        knobs = dict(zip(("leaf_cap", "group_cap", "walk_warps", "walk_stack"), (int(x) for x in t.tolist())))
        sim.close()
        sim = Simulation("accurate", "mixed", theta=W["theta"], eps=W["eps"], device=local, **knobs)
        sim.upload(bodies)
        attach(sim)
        sim.step(W["dt"])
    # warm-up (capacities, force cache, clocks)
    for _ in range(args.warmup):
        sim.step(W["dt"])
    sim.sync()
    # force error vs FP64 direct summation at the current positions
    idx = np.random.default_rng(12345).choice(n, min(4096, n), replace=False)
    a_mixed = sim.accel()
    d_direct = None
    state0 = None                           # the state d_direct belongs to: every leg's error is taken there
    if offsets is None:
        d_direct = sim.direct_accel(idx)
        err_mixed = force_error(a_mixed, d_direct, idx)
        state0 = dict(bodies)
        state0.update(sim.download())
    else:
        now = dict(bodies)
        now.update(sim.download())          # the direct sums must see the current positions
        err_mixed = ensemble_error(now, offsets, a_mixed, W, local)
    diag0 = sim.diagnostics()
    # ---- timed region: K steps, L2 flushed between steps, CUDA events per stage
    sim.reset_timers()
    sim.set_timing(True)
    launches0 = lib.next_kernel_launches()
    if dist:
        dist.barrier()
    sim.sync()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            sim.flush_l2()
            sim.steps(W["dt"], 1)       # one replay of the captured KDK-step graph
        sim.sync()
    if dist:
        dist.barrier()
    launches = lib.next_kernel_launches() - launches0   # the L2 flushes are memsets, not kernels
    sim.set_timing(False)
    st = sim.stats()
    if st["device_error"]:
        raise RuntimeError(f"device error word {st['device_error']} during the timed steps")
    ms_total = st["ms_step"]
    if dist:
        import torch
        t = torch.tensor([ms_total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    if dist:
        import torch
        tot = torch.tensor([float(st["pp_interactions"]), float(st["pc_interactions"]), st["ms_walk"]],
                           device=f"cuda:{local}", dtype=torch.float64)
        mx = tot[2:].clone()
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        st["pp_interactions"], st["pc_interactions"] = int(tot[0].item()), int(tot[1].item())
        st["ms_walk"] = float(mx[0].item())
    clocks = clk.summary()
    diag1 = sim.diagnostics()
    e0 = diag0["kinetic"] + diag0["potential"]
    e1 = diag1["kinetic"] + diag1["potential"]
    # sharded: every rank advances the same n bodies; independent systems: n is this rank's part
    total_bodies = n if sharded else world * n if world > 1 else n
    if world > 1 and not sharded:
        import torch
        tb = torch.tensor([float(n)], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tb, op=dist.ReduceOp.SUM)
        total_bodies = int(tb.item())
    value = total_bodies * args.steps / (ms_total * 1e-3)
    walk_ms = st["ms_walk"] / max(1, st["walk_launches"])
    flops_walk = (FLOPS_PP * st["pp_interactions"] + FLOPS_PC * st["pc_interactions"]) / max(1, st["walk_launches"])
    if sharded:
        flops_walk /= world          # per GPU: the interaction counts above are summed over ranks
    peak = fp32_peak(local)
    achieved = flops_walk / (walk_ms * 1e-3) / 1e12
    # ---- the same steps launched eagerly (no graph), CUDA-event timed
    sim.reset_timers()
    sim.set_timing(True)
    for _ in range(args.steps):
        sim.flush_l2()
        sim.step(W["dt"])
    sim.sync()
    eager_ms = sim.stats()["ms_step"]
    sim.set_timing(False)
    fp64 = None
    fp64g = None
    if rank == 0 and not args.skip_fp64:
        fp64 = plain_fp64_leg(bodies, offsets, W, local, max(1, args.fp64_steps), idx)
        if world == 1:
            fp64g = fp64_group_leg(state0 if state0 is not None else bodies, offsets, W, local,
                                   max(3, args.steps // 4), idx, d_direct, sim.get_params())
    # the reference's as-shipped forces on the same sampled bodies, same state
    cpu_accel = None
    if rank == 0 and state0 is not None and not args.skip_cpu and n <= 2_000_000:
        from oracle.oracle import Reference
        cpu_accel = Reference().accel_sample(state0, idx)
    refphys = None
    if rank == 0 and state0 is not None and world == 1 and not args.skip_fp64:
        refphys = ref_physics_leg(state0, W, local, max(1, args.fp64_steps), idx, d_direct, cpu_accel)
    big_sort = None
    if rank == 0 and world == 1 and args.config == "c2" and not args.skip_large_sort:
        big_sort = large_sort_leg(W, local)
    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if rank == 0 and not args.skip_e2e and offsets is None and world == 1:
        import ctypes as C
        ptrs = [lib.next_host_alloc(8 * n) for _ in range(7)]
        lanes = [np.ctypeslib.as_array(C.cast(p_, C.POINTER(C.c_double)), shape=(n,)) for p_ in ptrs]
        names = ("x", "y", "z", "vx", "vy", "vz")
        sim.download({k: lanes[i] for i, k in enumerate(names)})
        lanes[6][:] = bodies["m"]
        e_steps = max(3, args.steps // 4)
        for _ in range(2):                  # warm-up: the per-parity graph captures, first buffers
            sim.step_host(lanes, W["dt"])
        sim.sync()
        t0 = time.perf_counter()
        for _ in range(e_steps):
            sim.step_host(lanes, W["dt"])
        te = time.perf_counter() - t0
        e2e = {"value": n * e_steps / te, "unit": "particle-steps/s", "h2d_bytes_per_step": 7 * 8 * n,
               "d2h_bytes_per_step": 6 * 8 * n, "steps": e_steps,
               "path": "next_step_host on pinned host arrays per step (the reference's Step(): all seven input lanes "
                       "uploaded every call, KDK step, positions and velocities copied back), host wall clock after "
                       "2 untimed calls; the step starts on the held state while the upload lands and the upload is "
                       "checked bit for bit against the previous call's results (a mismatch re-runs the step)"}
        for p_ in ptrs:
            lib.next_host_free(p_)
    # ---- CPU baseline: the reference's own Step() on the host cores
    cpu = None
    if rank == 0 and not args.skip_cpu:
        if offsets is None and n <= 2_000_000:
            cpu = time_cpu_reference(bodies, W["dt"], args.cpu_budget)
            if cpu_accel is not None:
                cpu["force_error"] = force_error(cpu_accel, d_direct, np.arange(idx.shape[0]))
                cpu["force_error"]["versus"] = (f"FP64 direct summation with Plummer eps {W['eps']} on the same "
                                                f"{idx.shape[0]} sampled bodies (the reference's own softening differs)")
        else:
            cpu = {"skipped": "one reference Step() at this size takes minutes on the host; see the c2 line"}
    prm = sim.get_params()
    sim.close()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    peaks = measured_peaks()
    passes = sort_passes(st["key_levels"], 1 if offsets is None else len(offsets) - 1)
    sort_bpb = sort_bytes_per_body(passes)
    sort_gbs = sort_bpb * total_bodies / (st["ms_sort"] / args.steps * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
        "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32 interactions / f64 state",
        "data": "synthetic",
        "config": {"workload": W["name"], "n_bodies": n, "n_systems": 1 if offsets is None else len(offsets) - 1,
                   "theta": W["theta"], "eps": W["eps"], "dt": W["dt"], "seed": W["seed"],
                   "physics": "accurate (Plummer eps, full-width theta, corrected quadrupole)",
                   "precision": "FP32-mixed", "leaf_cap": prm.leaf_cap, "group_cap": prm.group_cap,
                   "walk_warps": prm.walk_warps, "walk_stack": prm.walk_stack,
                   "autotuned": tune is not None,
                   "parallelism": (f"sharded x{world}: force walk split by body share, NCCL all-gather of forces"
                                   if sharded else f"{world} ranks x independent systems" if world > 1 else "1 GPU"),
                   "l2": "flushed between steps (256 MiB write outside the timed events); step working set > L2"},
        "force_error": {"mixed": err_mixed, "fp64_plain": fp64["force_error"] if fp64 else None,
                        "versus": "FP64 direct summation on seeded bodies"},
        "fp64_gpu": fp64,
        "speedup_vs_fp64_gpu": value / fp64["value"] if fp64 and world == 1 else None,
        "fp64_same_structure_gpu": fp64g,
        "speedup_vs_fp64_same_structure": value / fp64g["value"] if fp64g else None,
        "ref_physics_fp64_gpu": refphys,
        "eager_value": total_bodies * args.steps / (eager_ms * 1e-3) if eager_ms else None,
        "step_launch": "one CUDA-graph replay per KDK step (captured kick-drift + force phase + kick)",
        "interactions_per_s": (st["pp_interactions"] + st["pc_interactions"]) / (st["ms_walk"] * 1e-3),
        "interactions_per_body": (st["pp_interactions"] + st["pc_interactions"]) / max(1, st["walk_launches"]) / total_bodies,
        "pp_fraction": st["pp_interactions"] / max(1, st["pp_interactions"] + st["pc_interactions"]),
        "pp_interactions_per_s": st["pp_interactions"] / (st["ms_walk"] * 1e-3),
        "pc_interactions_per_s": st["pc_interactions"] / (st["ms_walk"] * 1e-3),
        # the key sort's algorithmic traffic: passes x (12 B read + 12 B written) + the
        # 8-byte histogram read, per body, over the bench's own sort stage time;
        # passes = ceil(key bits / 8) of this run's keys (trimmed to the tree depth)
        "sort_hbm": {"passes": passes, "key_levels": st["key_levels"], "bytes_per_body": sort_bpb,
                     "gbs": sort_gbs, "frac": sort_gbs / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None,
                     "l2_resident": 2 * 24 * total_bodies < L2_BYTES,
                     "note": ("ping-pong buffers fit in the L2: not an HBM figure (see sort_hbm_large)"
                              if 2 * 24 * total_bodies < L2_BYTES else "buffers exceed the L2")},
        "sort_hbm_large": big_sort,
        "tree": {"nodes": st["n_nodes"], "internal": st["n_internal"], "groups": st["n_groups"] - st["n_systems"],
                 "bodies_per_group": n / max(1, st["n_groups"] - st["n_systems"]), "max_walk_stack": st["max_stack"]},
        "stage_ms_per_step": {"build": st["ms_build"] / args.steps, "sort": st["ms_sort"] / args.steps,
                              "walk": st["ms_walk"] / args.steps, "other": st["ms_other"] / args.steps},
        "energy_drift": abs(e1 - e0) / abs(e0),
        "autotune": tune,
        "roofline": {"bound": "fp32", "kernel": "walk_group_kernel<MixedArith<1,1,0>>", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "traffic": WALK_DRAM_BYTES if args.config == "c2" else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch of this workload "
                                       "(profiles/walk_group_mixed_cold_collapse_1M.md)",
                     "peak_source": "measured live by next_fp32_peak (FFMA chains); MEASURED_PEAKS.json has no FP32 entry",
                     "flops_per_launch": flops_walk, "ms_per_launch": walk_ms,
                     "flops_rule": "20 per body-body + 56 per body-cell interaction"},
        "hbm_peak_gbs": peaks.get("hbm_gbs"),
        "clocks": clocks,
        "gpu_launches": int(launches),
        "cpu_baseline": cpu,
        "e2e": e2e,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-large-sort", action="store_true")
    ap.add_argument("--full-run", action="store_true",
                    help="integrate the config's whole run (its step count) and report drift, not the bench line")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64group"], help="with --full-run")
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS), help="workload (default c2, the metric's)")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--n", type=int, default=None, help="override the body count of a single-system config")
    ap.add_argument("--leaf-cap", type=int, default=None, help="bodies per leaf of the mixed walk's tree")
    ap.add_argument("--group-cap", type=int, default=None, help="bodies per walk group (<= 32)")
    ap.add_argument("--walk-warps", type=int, default=None, help="warps per block of the mixed walk")
    ap.add_argument("--walk-stack", type=int, default=None, help="per-warp traversal stack entries")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.full_run:
        return full_run(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
