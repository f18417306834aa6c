"""Seeded synthetic initial conditions for the gravity workloads.

Every generator returns a dict of float64 numpy arrays ``x y z vx vy vz m``
plus an int32 ``type`` array (all zeros: every body is a type-0 body), in
G = 1 units.  The same seed always gives the same bodies.

* :func:`plummer`       -- Plummer sphere, inverse-CDF radii truncated at
  ``rmax`` scale radii, speeds by von Neumann rejection on
  g(q) = q^2 (1 - q^2)^3.5 (Aarseth, Henon & Wielen 1974).
* :func:`uniform_sphere` -- cold uniform-density sphere (cold collapse).
* :func:`hernquist`     -- Hernquist (1990) halo, inverse-CDF radii truncated
  at ``rmax`` scale radii, isotropic speeds sampled from the Eddington
  distribution function f(E) (Hernquist 1990, eq. 17).
* :func:`two_galaxies`  -- two disk + bulge + halo galaxies on a parabolic
  orbit.
* :func:`ensemble`      -- many independent Plummer spheres of uneven size.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["plummer", "uniform_sphere", "hernquist", "two_galaxies", "ensemble",
           "to_text", "from_text"]


def _isotropic(rng: np.random.Generator, r: np.ndarray):
    cos_t = rng.uniform(-1.0, 1.0, r.shape[0])
    sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    phi = rng.uniform(0.0, 2.0 * math.pi, r.shape[0])
    return r * sin_t * np.cos(phi), r * sin_t * np.sin(phi), r * cos_t


def _bodies(x, y, z, vx, vy, vz, m):
    n = x.shape[0]
    return {
        "x": np.ascontiguousarray(x, dtype=np.float64),
        "y": np.ascontiguousarray(y, dtype=np.float64),
        "z": np.ascontiguousarray(z, dtype=np.float64),
        "vx": np.ascontiguousarray(vx, dtype=np.float64),
        "vy": np.ascontiguousarray(vy, dtype=np.float64),
        "vz": np.ascontiguousarray(vz, dtype=np.float64),
        "m": np.ascontiguousarray(m, dtype=np.float64),
        "type": np.zeros(n, dtype=np.int32),
    }


def _plummer_radii(rng, n, a, rmax):
    out = np.empty(0)
    while out.shape[0] < n:
        u = rng.uniform(0.0, 1.0, int((n - out.shape[0]) * 1.05) + 16)
        u = u[u > 0.0]
        r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        out = np.concatenate([out, r[r < rmax * a]])
    return out[:n]


def _aarseth_q(rng, n):
    """q = v / v_escape with density g(q) = q^2 (1-q^2)^3.5 (max 0.0920 < 0.1)."""
    out = np.empty(0)
    while out.shape[0] < n:
        k = int((n - out.shape[0]) * 1.2) + 64
        q = rng.uniform(0.0, 1.0, k)
        y = rng.uniform(0.0, 0.1, k)
        ok = y < q * q * (1.0 - q * q) ** 3.5
        out = np.concatenate([out, q[ok]])
    return out[:n]


def plummer(n: int, seed: int = 0, a: float = 1.0, mass: float = 1.0, rmax: float = 20.0,
            rng: np.random.Generator | None = None):
    """Plummer sphere of ``n`` equal-mass bodies (total ``mass``, scale ``a``)."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    r = _plummer_radii(rng, n, a, rmax)
    x, y, z = _isotropic(rng, r)
    q = _aarseth_q(rng, n)
    # escape speed sqrt(2 G M / a) (1 + r^2/a^2)^(-1/4)
    v = q * math.sqrt(2.0 * mass / a) * (1.0 + (r / a) ** 2) ** (-0.25)
    vx, vy, vz = _isotropic(rng, v)
    return _bodies(x, y, z, vx, vy, vz, np.full(n, mass / n))


def uniform_sphere(n: int, seed: int = 1, radius: float = 1.0, mass: float = 1.0):
    """Cold (zero-velocity) uniform sphere of ``n`` equal-mass bodies."""
    rng = np.random.default_rng(seed)
    r = radius * rng.uniform(0.0, 1.0, n) ** (1.0 / 3.0)
    x, y, z = _isotropic(rng, r)
    zero = np.zeros(n)
    return _bodies(x, y, z, zero, zero, zero, np.full(n, mass / n))


def _hernquist_df(eps_rel, mass, a):
    """Isotropic Hernquist DF f(eps) for relative energy eps in (0, GM/a), G = 1."""
    vg = math.sqrt(mass / a)
    q = np.sqrt(np.clip(eps_rel * a / mass, 0.0, 1.0 - 1e-15))
    q2 = q * q
    pre = mass / (8.0 * math.sqrt(2.0) * math.pi ** 3 * a ** 3 * vg ** 3)
    body = 3.0 * np.arcsin(q) + q * np.sqrt(1.0 - q2) * (1.0 - 2.0 * q2) * (8.0 * q2 * q2 - 8.0 * q2 - 3.0)
    return pre * body / (1.0 - q2) ** 2.5


def _hernquist_speeds(rng, r, mass, a):
    """Speeds at radii r from p(v) ~ v^2 f(Psi - v^2/2) by rejection under a tabulated bound."""
    psi = mass / (r + a)
    vesc = np.sqrt(2.0 * psi)
    # Tabulate max_v v^2 f on a radius grid; bound each body by the larger of
    # the two bracketing grid values times a margin.
    lr = np.log(np.maximum(r, 1e-12))
    grid = np.linspace(lr.min() - 1e-9, lr.max() + 1e-9, 257)
    rg = np.exp(grid)
    psig = mass / (rg + a)
    t = np.linspace(0.0, 1.0, 2049)[1:-1]
    vv = np.sqrt(2.0 * psig)[:, None] * t[None, :]
    gg = vv * vv * _hernquist_df(psig[:, None] - 0.5 * vv * vv, mass, a)
    gmax = gg.max(axis=1)
    idx = np.clip(np.searchsorted(grid, lr) - 1, 0, grid.shape[0] - 2)
    bound = 1.2 * np.maximum(gmax[idx], gmax[idx + 1])
    out = np.empty_like(r)
    todo = np.arange(r.shape[0])
    while todo.shape[0]:
        v = rng.uniform(0.0, 1.0, todo.shape[0]) * vesc[todo]
        g = v * v * _hernquist_df(psi[todo] - 0.5 * v * v, mass, a)
        ok = rng.uniform(0.0, 1.0, todo.shape[0]) * bound[todo] < g
        out[todo[ok]] = v[ok]
        todo = todo[~ok]
    return out


def hernquist(n: int, seed: int = 4, a: float = 1.0, mass: float = 1.0, rmax: float = 50.0,
              rng: np.random.Generator | None = None):
    """Hernquist halo with isotropic Eddington-DF velocities."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    r = np.empty(0)
    while r.shape[0] < n:
        s = np.sqrt(rng.uniform(0.0, 1.0, int((n - r.shape[0]) * 1.05) + 16))
        s = s[s < 1.0]
        rr = a * s / (1.0 - s)
        r = np.concatenate([r, rr[rr < rmax * a]])
    r = r[:n]
    x, y, z = _isotropic(rng, r)
    v = _hernquist_speeds(rng, r, mass, a)
    vx, vy, vz = _isotropic(rng, v)
    return _bodies(x, y, z, vx, vy, vz, np.full(n, mass / n))


def _galaxy(rng, n, mass):
    """Exponential disk (60%), Plummer bulge a=0.2 (10%), Hernquist halo a=5 (30%)."""
    nd = int(round(0.6 * n))
    nb = int(round(0.1 * n))
    nh = n - nd - nb
    md, mb, mh = mass * nd / n, mass * nb / n, mass * nh / n
    # disk: R from the exponential surface density (scale 1), sech^2 layers (scale 0.1)
    R = -np.log(rng.uniform(1e-300, 1.0, nd) * rng.uniform(1e-300, 1.0, nd))
    phi = rng.uniform(0.0, 2.0 * math.pi, nd)
    zd = 0.1 * np.arctanh(rng.uniform(-1.0 + 1e-12, 1.0 - 1e-12, nd))
    xd, yd = R * np.cos(phi), R * np.sin(phi)
    rs = np.sqrt(R * R + zd * zd)
    menc = (md * (1.0 - (1.0 + R) * np.exp(-R))
            + mb * rs ** 3 / (rs * rs + 0.04) ** 1.5
            + mh * rs * rs / (rs + 5.0) ** 2)
    vc = np.sqrt(menc / np.maximum(rs, 1e-6))
    vxd, vyd, vzd = -vc * np.sin(phi), vc * np.cos(phi), np.zeros(nd)
    bulge = plummer(nb, a=0.2, mass=mb, rmax=20.0, rng=rng)
    halo = hernquist(nh, a=5.0, mass=mh, rmax=50.0, rng=rng)
    cat = lambda k, d: np.concatenate([d, bulge[k], halo[k]])
    return {
        "x": cat("x", xd), "y": cat("y", yd), "z": cat("z", zd),
        "vx": cat("vx", vxd), "vy": cat("vy", vyd), "vz": cat("vz", vzd),
        "m": np.concatenate([np.full(nd, md / max(nd, 1)), bulge["m"], halo["m"]]),
    }


def two_galaxies(n_per: int, seed: int = 2, separation: float = 30.0, pericentre: float = 5.0):
    """Two unit-mass galaxies ``separation`` apart on a parabolic orbit."""
    rng = np.random.default_rng(seed)
    g1, g2 = _galaxy(rng, n_per, 1.0), _galaxy(rng, n_per, 1.0)
    # tilt the second disk by 60 degrees about the x axis
    c, s = math.cos(math.pi / 3.0), math.sin(math.pi / 3.0)
    for p, q in (("y", "z"), ("vy", "vz")):
        a, b = g2[p].copy(), g2[q].copy()
        g2[p], g2[q] = c * a - s * b, s * a + c * b
    mtot = 2.0
    v = math.sqrt(2.0 * mtot / separation)
    vt = math.sqrt(2.0 * mtot * pericentre) / separation
    vr = -math.sqrt(max(v * v - vt * vt, 0.0))
    half = 0.5
    g1["x"] = g1["x"] - separation * half
    g2["x"] = g2["x"] + separation * half
    g1["vx"] = g1["vx"] - vr * half
    g2["vx"] = g2["vx"] + vr * half
    g1["vy"] = g1["vy"] - vt * half
    g2["vy"] = g2["vy"] + vt * half
    cat = lambda k: np.concatenate([g1[k], g2[k]])
    return _bodies(cat("x"), cat("y"), cat("z"), cat("vx"), cat("vy"), cat("vz"), cat("m"))


def ensemble(n_systems: int = 256, seed: int = 3, nmin: int = 1024, nmax: int = 65536):
    """Independent Plummer spheres with log-uniform sizes; returns (bodies, offsets).

    ``offsets`` has n_systems + 1 entries: system s owns bodies
    offsets[s] .. offsets[s+1]-1.
    """
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(nmin), math.log(nmax), n_systems)).astype(np.int64)
    parts = [plummer(int(k), rng=rng) for k in sizes]
    offsets = np.zeros(n_systems + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    cat = lambda k: np.concatenate([p[k] for p in parts])
    return _bodies(cat("x"), cat("y"), cat("z"), cat("vx"), cat("vy"), cat("vz"), cat("m")), offsets


def to_text(bodies, path):
    """Write the 8-column ``x y z vx vy vz m type`` text format at full precision."""
    cols = np.column_stack([bodies[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")])
    with open(path, "w") as f:
        for row, t in zip(cols, bodies["type"]):
            f.write(" ".join(repr(float(v)) for v in row) + " %d\n" % int(t))


def from_text(path):
    """Read the 8-column text format (stops at the first malformed row)."""
    rows = []
    with open(path) as f:
        toks = f.read().split()
    for i in range(0, len(toks) - 7, 8):
        try:
            rows.append([float(t) for t in toks[i:i + 7]] + [int(toks[i + 7])])
        except ValueError:
            break
    a = np.array(rows, dtype=np.float64).reshape(-1, 8)
    b = _bodies(a[:, 0], a[:, 1], a[:, 2], a[:, 3], a[:, 4], a[:, 5], a[:, 6])
    b["type"] = a[:, 7].astype(np.int32)
    return b
