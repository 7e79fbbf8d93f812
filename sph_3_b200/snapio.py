"""Raw binary initial-condition and snapshot files in the reference's layouts.

Three layouts, all little-endian, arrays stored one after the other:

* IC without header -- written by Evrard_Collapse_2024/IC_evrard.py:141-155
  and read by hfvGpuSphBHtree_newCool_v8_KH.cu:81-91 (N known from the
  file size, 44 bytes per particle):
      int32 Typ[N]; float32 x, y, z, vx, vy, vz, mass, h, eps, u  (each [N])
* IC with header -- read by readVectorsFromFile, hfvCLibs_v7_hfv_v8.1.h:58-103:
      int32 N; int32 Typ[N]; float32 x, y, z, vx, vy, vz, u, h, eps, mass
* snapshot -- written by saveArraysToBinary, hfvCLibs_v7_hfv_v8.1.h:110-141,
  read by pplot3.py:52-70:
      int32 N; int32 Typ[N]; float32 x, y, z, vx, vy, vz, rho, h, u, mass

Typ 0 marks gas particles; the SPH path here treats every particle as gas,
so loading a file with other types raises ValueError unless allowed.
"""
from __future__ import annotations

import numpy as np

IC_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "mass", "h", "eps", "u")
IC_HEADER_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "u", "h", "eps", "mass")
SNAP_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "rho", "h", "u", "mass")


def _to_state(d, allow_non_gas=False):
    typ = d["Typ"]
    if not allow_non_gas and np.any(typ != 0):
        raise ValueError("file holds non-gas particles (Typ != 0); pass allow_non_gas=True to load them as gas")
    out = {
        "pos": np.stack([d["x"], d["y"], d["z"]], axis=1).astype(np.float64),
        "vel": np.stack([d["vx"], d["vy"], d["vz"]], axis=1).astype(np.float64),
        "m": d["mass"].astype(np.float64),
        "Typ": typ,
    }
    for k in ("u", "h", "eps", "rho"):
        if k in d:
            out[k] = d[k].astype(np.float64)
    return out


def _read_blocks(buf, off, n, names):
    d = {}
    d["Typ"] = np.frombuffer(buf, dtype="<i4", count=n, offset=off).copy()
    off += 4 * n
    for name in names:
        d[name] = np.frombuffer(buf, dtype="<f4", count=n, offset=off).copy()
        off += 4 * n
    return d, off


def read_ic(path, allow_non_gas=False):
    """IC file without header (N from the file size)."""
    with open(path, "rb") as fh:
        buf = fh.read()
    if len(buf) % 44:
        raise ValueError("IC file size %d is not a multiple of 44 bytes" % len(buf))
    n = len(buf) // 44
    d, _ = _read_blocks(buf, 0, n, IC_FIELDS)
    return _to_state(d, allow_non_gas)


def read_ic_header(path, allow_non_gas=False):
    with open(path, "rb") as fh:
        buf = fh.read()
    n = int(np.frombuffer(buf, dtype="<i4", count=1)[0])
    if len(buf) != 4 + 44 * n:
        raise ValueError("header says N=%d but the file has %d bytes" % (n, len(buf)))
    d, _ = _read_blocks(buf, 4, n, IC_HEADER_FIELDS)
    return _to_state(d, allow_non_gas)


def read_snapshot(path, allow_non_gas=False):
    with open(path, "rb") as fh:
        buf = fh.read()
    n = int(np.frombuffer(buf, dtype="<i4", count=1)[0])
    if len(buf) != 4 + 44 * n:
        raise ValueError("header says N=%d but the file has %d bytes" % (n, len(buf)))
    d, _ = _read_blocks(buf, 4, n, SNAP_FIELDS)
    return _to_state(d, allow_non_gas)


def _columns(state, names, n):
    pos, vel = state["pos"], state.get("vel", np.zeros((n, 3)))
    cols = {"x": pos[:, 0], "y": pos[:, 1], "z": pos[:, 2], "vx": vel[:, 0], "vy": vel[:, 1], "vz": vel[:, 2],
            "mass": state["m"]}
    for k in ("u", "h", "eps", "rho"):
        cols[k] = state.get(k, np.zeros(n))
    return [np.ascontiguousarray(cols[k], dtype="<f4") for k in names]


def _write(path, state, names, header):
    n = state["pos"].shape[0]
    typ = np.ascontiguousarray(state.get("Typ", np.zeros(n, dtype=np.int32)), dtype="<i4")
    with open(path, "wb") as fh:
        if header:
            fh.write(np.array([n], dtype="<i4").tobytes())
        fh.write(typ.tobytes())
        for col in _columns(state, names, n):
            fh.write(col.tobytes())


def write_ic(path, state):
    _write(path, state, IC_FIELDS, header=False)


def write_ic_header(path, state):
    _write(path, state, IC_HEADER_FIELDS, header=True)


def write_snapshot(path, state):
    _write(path, state, SNAP_FIELDS, header=True)


def snapshot_of(ctx):
    """State dict of a Context in the snapshot's fields (caller's order)."""
    return {"pos": ctx.get_field("pos"), "vel": ctx.get_field("vel"), "rho": ctx.get_field("rho"),
            "h": ctx.get_field("h"), "u": ctx.get_field("u"), "m": ctx.get_field("m")}


def load_into(ctx, state):
    """Loads a state dict (from any reader) into a Context."""
    ctx.set_particles(state["pos"], state["m"], vel=state.get("vel"), u=state.get("u"),
                      h=state.get("h"), eps=state.get("eps"))
    return ctx
