"""One leapfrog KDK step of the reference's serial driver, composed from the
oracle functions -- test infrastructure only.

Order of operations follows sph_code/sph_serial.py:
  first step (lines 85-134): h bootstrap -> h search -> rho -> a_g -> P, c ->
      a_sph -> du/dt -> u += du/dt * dt (Euler), u_prev = u, ut_prev = du/dt
  loop body (lines 142-193): v += a dt/2; r += v dt; h; rho; a_g; P; c;
      du/dt (with the half-step v); u = u_prev + dt/2 (ut + ut_prev);
      a_sph (with P, c of the old u); a = a_g + a_sph; v += a dt/2.
The reference hard-codes N_ngb = 50 (+-5); ``n_ngb`` generalises it.
Gravity is the direct sum (``getAcc_g_smth_mpi`` row form).
"""
from __future__ import annotations

import numpy as np


def _p(params, key, default):
    return params.get(key, default) if params else default


def _forces(oc, st, params):
    gama = _p(params, "gamma", 5.0 / 3.0)
    alpha = _p(params, "alpha", 1.0)
    beta = _p(params, "beta", 2.0)
    eta = _p(params, "eta", 0.1)
    G = _p(params, "G", 1.0)
    n_ngb = _p(params, "n_ngb", 50)
    box = _p(params, "box", None)
    gravity = _p(params, "gravity", True)
    r, v, m, u = st["pos"], st["vel"], st["m"], st["u"]
    h, steps = oc.h_smooth_rows(r, st["h"], n_ngb=n_ngb, box=box)
    rho = oc.density_rows(r, m, h, box=box)
    if gravity:
        acc_g = oc.grav_direct_rows(r, m, G, st["eps"])
    else:
        acc_g = np.zeros_like(r)
    P = oc.getPressure(rho, u, gama)
    c = np.sqrt(gama * (gama - 1.0) * u)
    return dict(h=h, h_steps=steps, rho=rho, acc_g=acc_g, P=P, c=c, gama=gama, alpha=alpha,
                beta=beta, eta=eta, box=box)


def serial_first_step(oc, st, dt, params=None):
    """Initial forces and the Euler u update of sph_serial.py:85-134.

    ``st`` holds pos, vel, m, u, eps and (optionally) h; a missing h is
    bootstrapped with smoothing_length (k-th nearest distance / 2).
    Returns a new state dict with acc, u_prev, ut_prev, rho, P, c, h."""
    st = {k: (np.array(v, dtype=np.float64, copy=True) if isinstance(v, np.ndarray) else v)
          for k, v in st.items()}
    if st.get("h") is None:
        st["h"] = oc.smoothing_length_rows(st["pos"], k=_p(params, "n_boot", 50),
                                           box=_p(params, "box", None))
    f = _forces(oc, st, params)
    acc_sph, ut = oc.hydro_rows(st["pos"], st["vel"], f["rho"], f["P"], f["c"], f["h"], st["m"],
                                0, f["alpha"], f["beta"], f["eta"], box=f["box"])
    st["h"] = f["h"]
    st["rho"], st["P"], st["c"] = f["rho"], f["P"], f["c"]
    st["acc_g"], st["acc_sph"] = f["acc_g"], acc_sph
    st["acc"] = f["acc_g"] + acc_sph
    st["u"] = st["u"] + ut * dt
    st["u_prev"] = st["u"].copy()
    st["ut_prev"] = ut.copy()
    st["dudt"] = ut
    return st


def serial_step(oc, st, dt, params=None):
    """One loop iteration of sph_serial.py:142-196 on a copy of ``st``."""
    st = {k: (np.array(v, dtype=np.float64, copy=True) if isinstance(v, np.ndarray) else v)
          for k, v in st.items()}
    box = _p(params, "box", None)
    st["vel"] = st["vel"] + st["acc"] * dt / 2.0
    st["pos"] = st["pos"] + st["vel"] * dt
    if box is not None:
        b = np.asarray(box, dtype=np.float64)
        for k in range(3):
            if b[k] > 0:
                col = st["pos"][:, k]
                col[col < 0] += b[k]
                col[col >= b[k]] -= b[k]
    f = _forces(oc, st, params)
    _, ut = oc.hydro_rows(st["pos"], st["vel"], f["rho"], f["P"], f["c"], f["h"], st["m"], 0,
                          f["alpha"], f["beta"], f["eta"], box=box, want_acc=False)
    st["u"] = st["u_prev"] + 0.5 * dt * (ut + st["ut_prev"])
    st["u_prev"] = st["u"].copy()
    st["ut_prev"] = ut.copy()
    acc_sph, _ = oc.hydro_rows(st["pos"], st["vel"], f["rho"], f["P"], f["c"], f["h"], st["m"], 0,
                               f["alpha"], f["beta"], f["eta"], box=box, want_dudt=False)
    st["h"] = f["h"]
    st["rho"], st["P"], st["c"] = f["rho"], f["P"], f["c"]
    st["acc_g"], st["acc_sph"] = f["acc_g"], acc_sph
    st["acc"] = f["acc_g"] + acc_sph
    st["vel"] = st["vel"] + st["acc"] * dt / 2.0
    st["dudt"] = ut
    return st


# ------------------------------------------------------------------ MPI order
# sph_code/sph_mpi4_v4.py runs the same physics in another order and with
# the Balsara-switched ("shear") viscosity: the first step (lines 150-263)
# takes a_sph and du/dt with the same v; each loop iteration (lines 278-430)
# kicks and drifts, then h, rho, a_g, P, c (old u), div/curl v, a_sph, kicks
# with a = a_g + a_sph, and only then du/dt with the kicked v, followed by
# u = u_prev + dt/2 (du/dt + du/dt_prev).

def _shear(oc, st, f, want_acc, want_dudt, box):
    dv, cv = oc.div_curl_rows(st["pos"], st["vel"], f["rho"], st["m"], f["h"], box=box)
    acc, ut = oc.hydro_rows(st["pos"], st["vel"], f["rho"], f["P"], f["c"], f["h"], st["m"],
                            oc.VISC_BALSARA, f["alpha"], f["beta"], f["eta"], divV=dv, curlV=cv, box=box,
                            want_acc=want_acc, want_dudt=want_dudt)
    return acc, ut, dv, cv


def mpi4_first_step(oc, st, dt, params=None):
    """Initial forces and the Euler u update of sph_mpi4_v4.py:150-263."""
    st = {k: (np.array(v, dtype=np.float64, copy=True) if isinstance(v, np.ndarray) else v)
          for k, v in st.items()}
    if st.get("h") is None:
        st["h"] = oc.smoothing_length_rows(st["pos"], k=_p(params, "n_boot", 50),
                                           box=_p(params, "box", None))
    f = _forces(oc, st, params)
    acc_sph, ut, dv, cv = _shear(oc, st, f, True, True, f["box"])
    st["h"] = f["h"]
    st["rho"], st["P"], st["c"] = f["rho"], f["P"], f["c"]
    st["divV"], st["curlV"] = dv, cv
    st["acc_g"], st["acc_sph"] = f["acc_g"], acc_sph
    st["acc"] = f["acc_g"] + acc_sph
    st["u"] = st["u"] + ut * dt
    st["u_prev"] = st["u"].copy()
    st["ut_prev"] = ut.copy()
    st["dudt"] = ut
    return st


def mpi4_step(oc, st, dt, params=None):
    """One loop iteration of sph_mpi4_v4.py:278-430 on a copy of ``st``."""
    st = {k: (np.array(v, dtype=np.float64, copy=True) if isinstance(v, np.ndarray) else v)
          for k, v in st.items()}
    box = _p(params, "box", None)
    st["vel"] = st["vel"] + st["acc"] * dt / 2.0
    st["pos"] = st["pos"] + st["vel"] * dt
    f = _forces(oc, st, params)
    acc_sph, _, dv, cv = _shear(oc, st, f, True, False, box)
    st["acc_g"], st["acc_sph"] = f["acc_g"], acc_sph
    st["acc"] = f["acc_g"] + acc_sph
    st["vel"] = st["vel"] + st["acc"] * dt / 2.0
    _, ut = oc.hydro_rows(st["pos"], st["vel"], f["rho"], f["P"], f["c"], f["h"], st["m"],
                          oc.VISC_BALSARA, f["alpha"], f["beta"], f["eta"], divV=dv, curlV=cv, box=box,
                          want_acc=False)
    st["u"] = st["u_prev"] + 0.5 * dt * (ut + st["ut_prev"])
    st["u_prev"] = st["u"].copy()
    st["ut_prev"] = ut.copy()
    st["h"] = f["h"]
    st["rho"], st["P"], st["c"] = f["rho"], f["P"], f["c"]
    st["divV"], st["curlV"] = dv, cv
    st["dudt"] = ut
    return st
