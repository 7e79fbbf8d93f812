"""Physics validation of long Evrard runs against the 1-D PPM solution.

The reference checks its Evrard collapse runs by binning particles radially
and plotting the binned density, radial velocity and pressure over the PPM
profile (Particles_in_BH_Tree_III/Evrard_Collapse_2024/pplot3.py:12-49 loads
the profile, :100-200 bins and plots).  This module does the same as numbers:

* :func:`evolve` steps a context to a given time with a global time step
  dt_max / 2^k, k the smallest with dt at or below the smallest per-particle
  step of the reference's criterion (:meth:`Context.timestep`), re-evaluated
  every few steps (power-of-two steps keep the CUDA graph recaptures rare);
* :func:`radial_profile` bins density, radial velocity and pressure in
  logarithmic radial shells about the centre of mass (the reference's
  log-spaced grid);
* :func:`compare_ppm` interpolates a PPM profile at the shell centres and
  returns mean relative errors of density and pressure and the mean absolute
  error of the radial velocity over a radius range.

The PPM profile itself is data, passed in by the caller.
"""
from __future__ import annotations

import math

import numpy as np


def evolve(ctx, t_end, dt_max=1e-3, c_cfl=0.25, check_every=10, t0=0.0, first=True):
    """Steps ``ctx`` from t0 to t_end; returns (t, number of steps, dts used)."""
    t = float(t0)
    if first:
        # forces at t0 first, so that the start-up step already uses a safe dt
        passes = ["boot_h", "h", "density", "acc_sph", "dudt"] + (["gravity"] if ctx.config.gravity else [])
        ctx.compute(*passes)
        _, dtmin = ctx.timestep(c_cfl)
        k = 0 if not (dtmin < dt_max) else int(math.ceil(math.log2(dt_max / dtmin)))
        ctx.first_step(dt_max * 2.0 ** (-k))
    steps = 0
    used = []
    while t < t_end * (1 - 1e-12):
        _, dtmin = ctx.timestep(c_cfl)
        k = 0 if not (dtmin < dt_max) else int(math.ceil(math.log2(dt_max / dtmin)))
        dt = dt_max * 2.0 ** (-k)
        n = max(1, min(check_every, int((t_end - t) / dt)))
        if t + n * dt > t_end:
            dt = (t_end - t) / n
        ctx.step(dt, n)
        t += n * dt
        steps += n
        used.append(dt)
        status = ctx.status()
        if status:
            raise RuntimeError("device status during evolve: %s" % ctx.status_names())
    return t, steps, used


def radial_profile(pos, vel, rho, P, m=None, rmin=1e-3, rmax=1.5, nbins=100):
    """Mean density, radial velocity and pressure in log-spaced shells about
    the centre of mass; returns (r_mid, rho, v_r, P, count) for non-empty shells."""
    pos = np.asarray(pos, dtype=np.float64)
    vel = np.asarray(vel, dtype=np.float64)
    w = np.ones(len(pos)) if m is None else np.asarray(m, dtype=np.float64)
    com = (pos * w[:, None]).sum(0) / w.sum()
    vcom = (vel * w[:, None]).sum(0) / w.sum()
    x = pos - com
    v = vel - vcom
    r = np.linalg.norm(x, axis=1)
    vr = np.einsum("ij,ij->i", v, x) / np.maximum(r, 1e-300)
    grid = 10 ** np.linspace(np.log10(rmin), np.log10(rmax), nbins)
    idx = np.digitize(r, grid) - 1
    out = []
    for b in range(nbins - 1):
        sel = idx == b
        cnt = int(sel.sum())
        if cnt == 0:
            continue
        out.append((0.5 * (grid[b] + grid[b + 1]), rho[sel].mean(), vr[sel].mean(), P[sel].mean(), cnt))
    a = np.array(out)
    return a[:, 0], a[:, 1], a[:, 2], a[:, 3], a[:, 4].astype(int)


def compare_ppm(profile, ppm, r_lo=0.05, r_hi=0.8, min_count=20):
    """Errors of a radial profile against a PPM solution.

    ``profile`` is radial_profile's tuple; ``ppm`` a dict with radius, rho,
    press and vr arrays.  Returns mean |rho/rho_ppm - 1|, mean
    |P/P_ppm - 1| and mean |v_r - v_r,ppm| over shells with r_lo <= r <= r_hi
    and at least min_count particles, plus the number of shells used.
    """
    r, rho, vr, P, cnt = profile
    sel = (r >= r_lo) & (r <= r_hi) & (cnt >= min_count)
    lr = np.log(np.asarray(ppm["radius"], dtype=np.float64))
    rho_p = np.exp(np.interp(np.log(r[sel]), lr, np.log(ppm["rho"])))
    P_p = np.exp(np.interp(np.log(r[sel]), lr, np.log(ppm["press"])))
    v_p = np.interp(np.log(r[sel]), lr, ppm["vr"])
    return {"rho": float(np.mean(np.abs(rho[sel] / rho_p - 1))),
            "press": float(np.mean(np.abs(P[sel] / P_p - 1))),
            "vr": float(np.mean(np.abs(vr[sel] - v_p))),
            "shells": int(sel.sum())}
