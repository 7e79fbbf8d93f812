"""Seeded synthetic initial conditions for the benchmark and test workloads.

The reference's own IC files (pickles, raw .bin) are not in its repository,
so these generators stand in for them, following the recipes of its IC
scripts: an Evrard sphere with rho ~ 1/r (r = R sqrt(U), isotropic
directions, equal masses, u = 0.05 G M / R; cf. Evrard_Collapse_2024/IC_evrard.py,
which uses a stretched lattice instead of random radii), a jittered-lattice
Sedov blast in a periodic unit box, a density-contrast Kelvin-Helmholtz
slab, and a batch of Evrard clouds of log-uniform sizes.
"""
from __future__ import annotations

import numpy as np


def evrard(n, seed=0, M=1.0, R=1.0, u0=None, G=1.0):
    rng = np.random.default_rng(seed)
    r = R * np.sqrt(rng.random(n))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pos = d * r[:, None]
    m = np.full(n, M / n)
    vel = np.zeros((n, 3))
    u = np.full(n, 0.05 * G * M / R if u0 is None else u0)
    return dict(pos=pos, vel=vel, m=m, u=u)


def _m4(q):
    w = np.zeros_like(q)
    a = q <= 1.0
    b = (q > 1.0) & (q <= 2.0)
    w[a] = 1.0 - 1.5 * q[a] ** 2 + 0.75 * q[a] ** 3
    w[b] = 0.25 * (2.0 - q[b]) ** 3
    return w / np.pi


def sedov(n_side=128, seed=0, jitter=0.1, E=1.0, u_bg=1e-5, n_dep=64, box=1.0):
    """Jittered cubic lattice in the periodic box [0, box)^3, rho = 1, energy E
    deposited with M4 weights into the n_dep particles nearest the centre."""
    rng = np.random.default_rng(seed)
    dx = box / n_side
    g = (np.arange(n_side) + 0.5) * dx
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    pos += rng.normal(scale=jitter * dx, size=pos.shape)
    pos %= box
    n = pos.shape[0]
    m = np.full(n, box ** 3 / n)
    u = np.full(n, u_bg)
    c = np.full(3, 0.5 * box)
    r = np.linalg.norm(pos - c, axis=1)
    near = np.argsort(r, kind="stable")[:n_dep]
    h_dep = 0.5 * r[near].max() * 1.0000001
    w = _m4(r[near] / h_dep)
    u[near] += E * w / (w.sum() * m[near])
    return dict(pos=pos, vel=np.zeros((n, 3)), m=m, u=u, box=(box, box, box))


def kelvin_helmholtz(n=4194304, seed=0, P0=2.5, gamma=5.0 / 3.0, v0=0.5, amp=0.01):
    """Slab [0,1] x [0,1] x [0,1/16]: rho = 2 for |y - 0.5| < 0.25 else 1, on
    lattices whose spacing gives that density with equal masses; vx = +-v0,
    vy = amp sin(4 pi x); P = P0.  Exactly n particles (surplus lattice sites
    removed at random)."""
    rng = np.random.default_rng(seed)
    Lz = 1.0 / 16.0
    mass_tot = 2.0 * 0.5 * Lz + 1.0 * 0.5 * Lz
    m = mass_tot / n
    parts = []
    for rho, ylo, yhi in ((2.0, 0.25, 0.75), (1.0, 0.0, 0.25), (1.0, 0.75, 1.0)):
        d = (m / rho) ** (1.0 / 3.0)
        nx = int(np.ceil(1.0 / d))
        ny = int(np.ceil((yhi - ylo) / d))
        nz = int(np.ceil(Lz / d))
        gx = (np.arange(nx) + 0.5) * (1.0 / nx)
        gy = ylo + (np.arange(ny) + 0.5) * ((yhi - ylo) / ny)
        gz = (np.arange(nz) + 0.5) * (Lz / nz)
        X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
        parts.append(np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1))
    pos = np.concatenate(parts)
    if pos.shape[0] > n:
        keep = np.sort(rng.choice(pos.shape[0], n, replace=False))
        pos = pos[keep]
    elif pos.shape[0] < n:
        extra = rng.random((n - pos.shape[0], 3)) * np.array([1.0, 1.0, Lz])
        pos = np.concatenate([pos, extra])
    inner = np.abs(pos[:, 1] - 0.5) < 0.25
    rho = np.where(inner, 2.0, 1.0)
    vel = np.zeros((n, 3))
    vel[:, 0] = np.where(inner, v0, -v0)
    vel[:, 1] = amp * np.sin(4.0 * np.pi * pos[:, 0])
    u = P0 / ((gamma - 1.0) * rho)
    return dict(pos=pos, vel=vel, m=np.full(n, m), u=u, box=(1.0, 1.0, Lz))


def evrard_batch(ncloud=256, seed=0, n_min=2048, n_max=65536, mr_range=(0.5, 2.0)):
    """ncloud independent Evrard clouds, N log-uniform in [n_min, n_max], own
    M and R uniform in mr_range; returns the concatenation and the counts."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(n_min), np.log(n_max), ncloud)).astype(np.int64)
    Ms = rng.uniform(*mr_range, ncloud)
    Rs = rng.uniform(*mr_range, ncloud)
    out = {k: [] for k in ("pos", "vel", "m", "u")}
    for k in range(ncloud):
        ic = evrard(int(counts[k]), seed=seed * 100003 + k + 1, M=Ms[k], R=Rs[k])
        for key in out:
            out[key].append(ic[key])
    res = {k: np.concatenate(v) for k, v in out.items()}
    res["counts"] = counts
    res["M"] = Ms
    res["R"] = Rs
    return res
