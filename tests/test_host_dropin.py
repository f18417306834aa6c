"""The C++ drop-in layer: Particle / Step / computeAdaptiveDt headers and the `next` CLI.

CPU tests cover the CLI contract (argument count and format errors exit 1
before any device work).  GPU tests compile a reference-style main loop
against the drop-in headers and compare it with the reference's own Step()
trajectories (golden fixtures) and with the oracle.
"""
import os
import subprocess

import numpy as np
import pytest

from golden_cases import load
from next_b200 import ic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NEXT = os.path.join(ROOT, "next_b200", "bin", "next")
HOST = os.path.join(ROOT, "next_b200", "host")
LIB = os.path.join(ROOT, "next_b200", "lib")


def run_next(args, cwd, env=None, stdin=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([NEXT, *args], cwd=cwd, env=e, input=stdin, capture_output=True, text=True, timeout=300)


def test_cli_usage_and_format_errors(tmp_path):
    r = run_next([], tmp_path)
    assert r.returncode == 1 and "Usage: next" in r.stderr
    r = run_next(["ic.txt", "1", "0.001", "0.1", "png"], tmp_path)
    assert r.returncode == 1 and "Choose a file format" in r.stderr
    r = run_next(["ic.txt", "1", "0.001", "0.1", "hdf5"], tmp_path)
    assert r.returncode == 1 and "hdf5" in r.stderr


def test_text_loader_stops_at_first_malformed_row(tmp_path):
    b = ic.plummer(10, seed=1)
    p = tmp_path / "ic.txt"
    ic.to_text(b, p)
    with open(p, "a") as f:
        f.write("1 2 3 oops\n4 5 6 7 8 9 10 0\n")
    back = ic.from_text(p)
    assert back["x"].shape[0] == 10


@pytest.fixture(scope="module")
def snapshot_bin(tmp_path_factory):
    """The drop-in VTK/VTU writers (header-only, no GPU) in a small program."""
    out = tmp_path_factory.mktemp("bin") / "save_snapshot"
    subprocess.run(["g++", "-O2", "-std=c++17", "-DNEXT_FP64", f"-I{HOST}",
                    os.path.join(ROOT, "tests", "cpp", "save_snapshot.cpp"), "-o", str(out)], check=True)
    return str(out)


@pytest.mark.parametrize("fmt", ["vtk", "vtu"])
def test_snapshot_bytes_equal_reference_writer(tmp_path, snapshot_bin, fmt):
    """SaveVTK / SaveVTU write the same bytes as the reference's own writers
    (src/io/vtk_save.h:21-75, src/io/vtu_save.h:22-78), NEXT_FP64 build."""
    from oracle.oracle import Reference
    rng = np.random.default_rng(31)
    n = 1000
    b = ic.plummer(n, seed=5)
    b["type"] = rng.integers(0, 2, n).astype(np.int32)
    b["m"][::97] = 0.0                                # zero masses print as "0"
    b["x"][3], b["vy"][4] = -1.25e-7, 3.5e12          # exponent formatting
    raw = tmp_path / "bodies.bin"
    with open(raw, "wb") as f:
        for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
            f.write(np.ascontiguousarray(b[k], dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(b["type"], dtype=np.int32).tobytes())
    mine, ref = tmp_path / f"mine.{fmt}", tmp_path / f"ref.{fmt}"
    subprocess.run([snapshot_bin, str(raw), str(n), fmt, str(mine)], check=True)
    Reference().save_snapshot(b, ref, fmt)
    assert mine.read_bytes() == ref.read_bytes()
    assert mine.stat().st_size > 60 * n


@pytest.fixture(scope="module")
def dropin_bin(tmp_path_factory):
    out = tmp_path_factory.mktemp("bin") / "dropin_step"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{HOST}", os.path.join(ROOT, "tests", "cpp", "dropin_step.cpp"),
                    f"-L{LIB}", "-lnext_b200", f"-Wl,-rpath,{LIB}", "-o", str(out)], check=True)
    return str(out)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["plummer1024_dm", "mixed_mass300", "two_body"])
def test_dropin_step_matches_reference(tmp_path, dropin_bin, name):
    b, z = load(name)
    p = tmp_path / "ic.txt"
    ic.to_text(b, p)
    r = subprocess.run([dropin_bin, str(p), repr(float(z["step_dt"])), str(int(z["nsteps"])), "0"],
                       capture_output=True, text=True, timeout=300, check=True)
    got = np.loadtxt(r.stdout.splitlines(), ndmin=2)
    want = np.column_stack([z["out_" + c] for c in ("x", "y", "z", "vx", "vy", "vz")])
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


@pytest.mark.gpu
def test_dropin_adaptive_loop_matches_oracle(tmp_path, dropin_bin, oracle):
    b = ic.plummer(2000, seed=13)
    b["type"][::3] = 1
    p = tmp_path / "ic.txt"
    ic.to_text(b, p)
    back = ic.from_text(p)
    r = subprocess.run([dropin_bin, str(p), "0.01", "5", "1"], capture_output=True, text=True, timeout=300,
                       check=True)
    got = np.loadtxt(r.stdout.splitlines(), ndmin=2)
    s = back
    for _ in range(5):
        s = oracle.step(s, oracle.adaptive_dt(s, 0.01), 1, mode="ref")
    want = np.column_stack([s[c] for c in ("x", "y", "z", "vx", "vy", "vz")])
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


@pytest.mark.gpu
def test_cli_runs_and_dumps(tmp_path, oracle):
    b = ic.plummer(1500, seed=14)
    ic.to_text(b, tmp_path / "ic.txt")
    back = ic.from_text(tmp_path / "ic.txt")
    # dump interval 0: a dump after every step, so dump_3 holds the state after 4 steps
    r = run_next(["ic.txt", "4", "0.01", "0", "vtk"], tmp_path, env={"NEXT_MAX_STEPS": "4"})
    assert r.returncode == 0, r.stderr
    assert "Particles: 1500" in r.stdout and "[Dump 0]" in r.stdout
    dumps = sorted(tmp_path.glob("dump_*.vtk"))
    assert len(dumps) == 4
    # last dump against the oracle's reference-physics loop
    s = back
    for _ in range(4):
        s = oracle.step(s, oracle.adaptive_dt(s, 0.01), 1, mode="ref")
    lines = open(tmp_path / "dump_3.vtk").read().splitlines()
    k = lines.index(next(l for l in lines if l.startswith("POINTS")))
    pts = np.array([[float(v) for v in l.split()] for l in lines[k + 1:k + 1 + 1500]])
    # default iostream formatting keeps 6 significant digits
    assert np.allclose(pts[:, 0], s["x"], rtol=1e-5, atol=1e-6)
    r = run_next(["ic.txt", "1", "0.01", "0.05", "vtu"], tmp_path, env={"NEXT_MAX_STEPS": "2"})
    assert r.returncode == 0 and (tmp_path / "dump_0.vtu").exists()
    r = run_next(["ic.txt", "1", "0.01", "1.0", "vtk"], tmp_path, stdin="q\n")
    assert r.returncode == 0 and "Exiting..." in r.stdout
