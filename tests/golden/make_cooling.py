"""Golden vectors for the heating/cooling step, from the reference's own GPU
kernel hcoolingZ (Particles_in_BH_Tree_III/Evrard_Collapse_2024/
hfvCLibs_v7_hfv_v8.1.h:1433-1623), in three stages:

    python tests/golden/make_cooling.py inputs -
        writes a seeded table in the layout of the reference's
        coolHeatGridJan2024.bin (the CHIMES tables are not distributed with
        the reference) and 4,096 seeded particles whose radii, densities and
        energies cover the table's grids, their edges and the space beyond
        them (plus 10 % non-gas particles, which the kernel leaves alone):
        oracle/_ref/cooling_in.npz and the kernel's input file
        oracle/_ref/cooling_in.bin;
    python tests/golden/make_cooling.py run OUT.bin
        (on a GPU) runs oracle/_ref/ref_cooling (oracle/build_ref.sh: the
        reference kernel, unchanged) on that input;
    python tests/golden/make_cooling.py merge OUT.bin
        writes cooling_ref.npz: the table, the inputs, and the kernel's new u
        and ion fractions.

The tests read only cooling_ref.npz.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
IN_NPZ = os.path.join(ROOT, "oracle", "_ref", "cooling_in.npz")
IN_BIN = os.path.join(ROOT, "oracle", "_ref", "cooling_in.bin")
OUT_NPZ = os.path.join(HERE, "cooling_ref.npz")

DIMS = (7, 20, 10, 3, 4, 8)  # N_kpc, N_T, N_nH, N_Z, N_M, N_t
# unit density (cgs), unit time (s), unit u (cgs), unit length (cm), kpc (cm)
UNITS = np.array([6.77e-23, 3.156e13, 1.0e10, 3.086e21, 3.086e21], np.float32)
DT = np.float32(2.0e-4)
N = 4096


def table(seed=5):
    rng = np.random.default_rng(seed)
    nk, nT, nh, nZ, nM, nt = DIMS
    kpc = np.array([0.0, 0.1, 0.25, 0.5, 1.0, 2.0, 4.0], np.float32)
    nH = np.float32(10.0) ** np.linspace(-3, 3, nh).astype(np.float32)
    T = np.float32(10.0) ** np.linspace(1, 8, nT).astype(np.float32)
    t = np.array([0.0, 1e6, 1e8, 1e9, 3e9, 1e10, 1e11, 1e12], np.float32)
    mu = np.float32(0.6) + np.float32(0.5) * rng.random((nk, 1, nh, nZ)).astype(np.float32)
    uarr = (np.float32(2.07e8) * T[None, :, None, None] / mu).astype(np.float32)  # 1.5 k T / (mu mH)
    ueq = uarr[:, 6:7] * (np.float32(1.0) + np.float32(0.5) * rng.random((nk, 1, nh, nZ)).astype(np.float32))
    tau = np.float32(1e9) / (np.float32(1.0) + nH[None, None, :, None]) * (np.float32(1.0) + rng.random((nk, nT, nh, nZ)).astype(np.float32))
    frac = np.exp(-t[None, None, None, None, :].astype(np.float64) / tau[..., None]).astype(np.float32)
    uevol = (ueq[..., None] + (uarr[..., None] - ueq[..., None]) * frac).astype(np.float32)
    # species fractions on a 1/256 lattice (the fixture compresses)
    metalz = (rng.integers(0, 256, (nk, nT, nh, nZ, nM, nt)) / np.float32(256.0)).astype(np.float32)
    return {"dims": np.array(DIMS, np.int32), "kpc": kpc, "nH": nH, "t": t, "uEvol": uevol,
            "metalz": metalz, "uArr": uarr}


def particles(tab, seed=6):
    rng = np.random.default_rng(seed)
    n = N
    # radii (code length = kpc) over [0, 5] kpc, some exactly on grid points
    r = rng.uniform(0.0, 5.0, n).astype(np.float32)
    r[:64] = np.resize(tab["kpc"], 64)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pos = (d * r[:, None]).astype(np.float32)
    # densities: nH from 1e-4 to 1e4 cm^-3 (beyond the grid both ways)
    nh = 10.0 ** rng.uniform(-4, 4, n)
    rho = (nh * 1.6726e-24 / 0.70 / UNITS[0]).astype(np.float32)
    # u: across the T grid, below its first row and above its last
    T = 10.0 ** rng.uniform(0.5, 8.5, n)
    u = (2.07e8 * T / 0.9 / UNITS[2]).astype(np.float32)
    typ = np.where(rng.random(n) < 0.1, 1, 0).astype(np.int32)
    return typ, u, rho, pos


def inputs(_unused="-"):
    tab = table()
    typ, u, rho, pos = particles(tab)
    os.makedirs(os.path.dirname(IN_BIN), exist_ok=True)
    np.savez_compressed(IN_NPZ, **tab, units=UNITS, dt=DT, typ=typ, u=u, rho=rho, pos=pos)
    with open(IN_BIN, "wb") as fh:
        np.array([N], np.int32).tofile(fh)
        np.concatenate([[DT], UNITS]).astype(np.float32).tofile(fh)
        tab["dims"].astype(np.int32).tofile(fh)
        for k in ("kpc", "nH", "t", "uEvol", "metalz", "uArr"):
            np.ascontiguousarray(tab[k], np.float32).tofile(fh)
        typ.tofile(fh)
        for a in (u, rho, pos[:, 0], pos[:, 1], pos[:, 2]):
            np.ascontiguousarray(a, np.float32).tofile(fh)
    print("wrote", IN_NPZ, IN_BIN)


def run(out_bin):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_cooling")
    subprocess.check_call([exe, IN_BIN, out_bin])


def merge(out_bin):
    d = dict(np.load(IN_NPZ))
    with open(out_bin, "rb") as fh:
        n, nm = (int(v) for v in np.fromfile(fh, dtype=np.int32, count=2))
        u_new = np.fromfile(fh, dtype=np.float32, count=n)
        ion = np.fromfile(fh, dtype=np.float32, count=n * nm).reshape(n, nm)
    assert n == d["u"].shape[0] and nm == int(d["dims"][4])
    d.update(u_new=u_new, ionfrac=ion)
    np.savez_compressed(OUT_NPZ, **d)
    print("wrote", OUT_NPZ)


if __name__ == "__main__":
    if len(sys.argv) < 3 or sys.argv[1] not in ("inputs", "run", "merge"):
        sys.exit(__doc__)
    {"inputs": inputs, "run": run, "merge": merge}[sys.argv[1]](sys.argv[2])
