"""The seeded initial-condition generators (next_b200/ic.py) against their models.

Every benchmark workload starts from these generators, so each is checked
against the analytic model it samples, at 200,000 bodies:

* radii: Kolmogorov-Smirnov test of the sampled radii against the model's
  cumulative mass profile, truncated where the generator truncates;
* velocities: kinetic energy T and potential energy W against the values the
  model gives for the truncated body distribution, T from the isotropic Jeans
  dispersion of the (untruncated) model whose distribution function the
  speeds are drawn from, W from the truncated mass profile; W of the sample
  is estimated from FP64 direct sums (the oracle) on 4096 sampled bodies;
* Plummer speeds: q = v / v_esc against Aarseth's g(q) = q^2 (1 - q^2)^3.5;
* the two-galaxy encounter: separation, parabolic relative orbit and its
  pericentre (point-mass two-body orbit), disk scale length and height;
* the ensemble: log-uniform system sizes in [1024, 65536], unit mass each.

Physics constants: G = 1, all bodies type 0.
"""
import math

import numpy as np
import pytest

from next_b200 import ic

integrate = pytest.importorskip("scipy.integrate")
stats = pytest.importorskip("scipy.stats")

N = 200_000


def _truncated_energies(rho, mass, rt):
    """(T, W) of a unit-mass body set drawn from density rho truncated at rt, with
    speeds from the isotropic distribution function of the untruncated model."""
    mt = mass(rt)

    def sigma2(r):   # isotropic Jeans equation of the untruncated model
        return integrate.quad(lambda s: rho(s) * mass(s) / s ** 2, r, np.inf, limit=200)[0] / rho(r)

    T = integrate.quad(lambda r: rho(r) / mt * 1.5 * sigma2(r) * 4 * np.pi * r * r, 0, rt, limit=200)[0]
    W = -integrate.quad(lambda r: (mass(r) / mt) * rho(r) / mt * 4 * np.pi * r, 0, rt, limit=200)[0]
    return T, W


def _sample_energies(oracle, b, k=4096, seed=0):
    n = b["x"].shape[0]
    idx = np.random.default_rng(seed).choice(n, k, replace=False)
    pot = oracle.direct(b, idx, eps=1e-4)["pot"]
    W = 0.5 * n / k * float(np.sum(b["m"][idx] * pot))
    T = 0.5 * float(np.sum(b["m"] * (b["vx"] ** 2 + b["vy"] ** 2 + b["vz"] ** 2)))
    return T, W


def _radii(b, centre=(0.0, 0.0, 0.0)):
    return np.sqrt((b["x"] - centre[0]) ** 2 + (b["y"] - centre[1]) ** 2 + (b["z"] - centre[2]) ** 2)


RHO_PLUMMER = lambda r: 3.0 / (4.0 * np.pi) * (1.0 + r * r) ** -2.5
M_PLUMMER = lambda r: r ** 3 / (1.0 + r * r) ** 1.5
RHO_HERNQUIST = lambda r: 1.0 / (2.0 * np.pi) / (r * (1.0 + r) ** 3)
M_HERNQUIST = lambda r: r * r / (1.0 + r) ** 2


@pytest.fixture(scope="module")
def plummer():
    return ic.plummer(N, seed=0)


@pytest.fixture(scope="module")
def hernquist():
    return ic.hernquist(N, seed=4)


def test_generators_are_seeded():
    a, b = ic.plummer(1000, seed=7), ic.plummer(1000, seed=7)
    assert all(np.array_equal(a[k], b[k]) for k in a)
    c = ic.plummer(1000, seed=8)
    assert not np.array_equal(a["x"], c["x"])
    assert a["type"].dtype == np.int32 and not a["type"].any()


def test_plummer_mass_profile(plummer):
    r = _radii(plummer)
    assert r.max() < 20.0 and abs(plummer["m"].sum() - 1.0) < 1e-12
    cdf = lambda x: M_PLUMMER(np.minimum(x, 20.0)) / M_PLUMMER(20.0)
    assert stats.kstest(r, cdf).pvalue > 1e-3


def test_plummer_aarseth_speeds(plummer):
    r = _radii(plummer)
    v = np.sqrt(plummer["vx"] ** 2 + plummer["vy"] ** 2 + plummer["vz"] ** 2)
    q = v / (math.sqrt(2.0) * (1.0 + r * r) ** -0.25)
    assert q.max() < 1.0
    norm = integrate.quad(lambda s: s * s * (1 - s * s) ** 3.5, 0, 1)[0]
    cdf = np.vectorize(lambda x: integrate.quad(lambda s: s * s * (1 - s * s) ** 3.5, 0, min(max(x, 0.0), 1.0))[0] / norm)
    assert stats.kstest(q[:20_000], cdf).pvalue > 1e-3
    # isotropy: no preferred direction of the velocities
    for c in ("vx", "vy", "vz"):
        assert abs(np.mean(plummer[c])) < 5 * np.std(plummer[c]) / math.sqrt(N)


def test_plummer_virial(oracle, plummer):
    T, W = _sample_energies(oracle, plummer)
    Te, We = _truncated_energies(RHO_PLUMMER, M_PLUMMER, 20.0)
    assert abs(T / Te - 1) < 0.015 and abs(W / We - 1) < 0.02
    assert abs(2 * T / abs(W) - 1.0) < 0.02          # in equilibrium


def test_hernquist_mass_profile(hernquist):
    r = _radii(hernquist)
    assert r.max() < 50.0 and abs(hernquist["m"].sum() - 1.0) < 1e-12
    cdf = lambda x: M_HERNQUIST(np.minimum(x, 50.0)) / M_HERNQUIST(50.0)
    assert stats.kstest(r, cdf).pvalue > 1e-3


def test_hernquist_eddington_speeds(oracle, hernquist):
    T, W = _sample_energies(oracle, hernquist)
    Te, We = _truncated_energies(RHO_HERNQUIST, M_HERNQUIST, 50.0)
    assert abs(T / Te - 1) < 0.015 and abs(W / We - 1) < 0.02
    # the dispersion profile follows the model's Jeans solution bin by bin
    r = _radii(hernquist)
    v2 = hernquist["vx"] ** 2 + hernquist["vy"] ** 2 + hernquist["vz"] ** 2
    edges = np.quantile(r, np.linspace(0.05, 0.95, 10))
    for lo, hi in zip(edges[:-1], edges[1:]):
        sel = (r >= lo) & (r < hi)
        rm = float(np.median(r[sel]))
        s2 = integrate.quad(lambda s: RHO_HERNQUIST(s) * M_HERNQUIST(s) / s ** 2, rm, np.inf, limit=200)[0] / RHO_HERNQUIST(rm)
        assert abs(np.mean(v2[sel]) / (3 * s2) - 1) < 0.06, (lo, hi)


def test_uniform_sphere_is_cold_and_uniform():
    b = ic.uniform_sphere(N, seed=1)
    r = _radii(b)
    assert r.max() <= 1.0 and not (b["vx"].any() or b["vy"].any() or b["vz"].any())
    assert stats.kstest(r, lambda x: np.clip(x, 0, 1) ** 3).pvalue > 1e-3
    # isotropic directions: cos(theta) uniform in [-1, 1]
    assert stats.kstest(b["z"] / r, "uniform", args=(-1, 2)).pvalue > 1e-3


def test_two_galaxy_parabolic_orbit():
    n_per = N // 2
    b = ic.two_galaxies(n_per, seed=2)
    m = b["m"]
    halves = (slice(0, n_per), slice(n_per, 2 * n_per))
    com = [np.array([np.sum(m[s] * b[k][s]) / np.sum(m[s]) for k in ("x", "y", "z")]) for s in halves]
    vel = [np.array([np.sum(m[s] * b[k][s]) / np.sum(m[s]) for k in ("vx", "vy", "vz")]) for s in halves]
    mass = [float(np.sum(m[s])) for s in halves]
    assert all(abs(mm - 1.0) < 1e-9 for mm in mass)
    d = com[1] - com[0]
    v = vel[1] - vel[0]
    sep = float(np.linalg.norm(d))
    assert abs(sep - 30.0) < 0.5
    # relative orbit of two point masses: parabolic (E = 0) with pericentre 5
    mu, mt = mass[0] * mass[1] / (mass[0] + mass[1]), mass[0] + mass[1]
    kin = 0.5 * mu * float(v @ v)
    energy = kin - mass[0] * mass[1] / sep
    assert abs(energy) < 0.05 * kin
    h = float(np.linalg.norm(np.cross(d, v)))
    assert abs(h * h / (2.0 * mt) / 5.0 - 1.0) < 0.05
    # approaching, total momentum zero
    assert float(d @ v) < 0
    assert np.linalg.norm(mass[0] * vel[0] + mass[1] * vel[1]) < 0.01 * np.linalg.norm(v)


def test_galaxy_components():
    n = N // 2
    g = ic.two_galaxies(n, seed=2)
    nd = int(round(0.6 * n))
    x0 = -15.0                                       # first galaxy, untilted disk
    R = np.sqrt((g["x"][:nd] - x0) ** 2 + g["y"][:nd] ** 2)
    # exponential disk: scale length 1 (enclosed fraction 1 - (1 + R) e^-R), sech^2 height 0.1
    assert stats.kstest(R, lambda x: 1 - (1 + x) * np.exp(-x)).pvalue > 1e-3
    assert stats.kstest(g["z"][:nd], lambda z: 0.5 * (1 + np.tanh(z / 0.1))).pvalue > 1e-3
    # masses: 60 / 10 / 30 % in disk / bulge / halo
    assert abs(np.sum(g["m"][:nd]) - 0.6) < 1e-9
    nb = int(round(0.1 * n))
    assert abs(np.sum(g["m"][nd:nd + nb]) - 0.1) < 1e-9


def test_ensemble_sizes_log_uniform():
    b, offsets = ic.ensemble(256, seed=3)
    sizes = np.diff(offsets)
    assert sizes.shape[0] == 256 and sizes.min() >= 1024 and sizes.max() <= 65536
    assert offsets[-1] == b["x"].shape[0]
    assert 3.0e6 < offsets[-1] < 6.5e6
    u = (np.log(sizes) - math.log(1024)) / (math.log(65536) - math.log(1024))
    assert stats.kstest(u, "uniform").pvalue > 1e-3
    for s in range(0, 256, 37):
        assert abs(np.sum(b["m"][offsets[s]:offsets[s + 1]]) - 1.0) < 1e-9
