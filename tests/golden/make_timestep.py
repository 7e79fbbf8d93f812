"""Golden vectors for the per-particle time-step criterion, from the
reference's own GPU kernel dt_array_indiv_dt
(Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1189-1262),
in three stages:

    python tests/golden/make_timestep.py inputs /path/to/reference
        (needs the reference checked out, numba) builds a consistent SPH state
        with the reference's own CPU functions (sph_code/libsx.py, shear.py):
        Evrard N = 2000 with random velocities, h from its h rule, rho,
        div v, c, gravity and hydro accelerations -- every kernel input
        rounded to float32 -- and writes oracle/_ref/timestep_in.npz and the
        kernel's input file oracle/_ref/timestep_in.bin;
    python tests/golden/make_timestep.py run OUT.bin
        (on a GPU) runs oracle/_ref/ref_timestep (oracle/build_ref.sh: the
        reference kernel, unchanged) on that input;
    python tests/golden/make_timestep.py merge OUT.bin
        writes timestep_ref.npz: the inputs and the kernel's float32 dt,
        dh/dt, |a_g| and |a_tot|.

The tests read only timestep_ref.npz.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
IN_NPZ = os.path.join(ROOT, "oracle", "_ref", "timestep_in.npz")
IN_BIN = os.path.join(ROOT, "oracle", "_ref", "timestep_in.bin")
OUT_NPZ = os.path.join(HERE, "timestep_ref.npz")
C_CFL, ALPHA = 0.25, 1.0
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "atx", "aty", "atz", "h", "c", "divV", "eps")


def inputs(ref_root, n=2000, seed=31):
    sys.path.insert(0, os.path.join(ref_root, "sph_code"))
    import libsx  # noqa: E402  (the reference)
    import shear  # noqa: E402  (the reference)
    sys.path.insert(0, ROOT)
    from sph_3_b200.ic import evrard
    ic = evrard(n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)  # noqa: E731
    pos = f32(ic["pos"])
    v = f32(rng.normal(scale=0.1, size=(n, 3)))
    m = ic["m"]
    u = 0.05 * (1.0 + 0.5 * rng.random(n))
    eps = f32(np.full(n, 0.01))
    gama = 5.0 / 3.0
    h = f32(libsx.h_smooth_fast(pos, libsx.smoothing_length_mpi(0, n, pos)))
    rho = libsx.getDensity(pos, m, h)
    divV, _ = shear.div_curlVel(pos, v, rho, m, h)
    c = np.sqrt(gama * (gama - 1.0) * u)
    P = libsx.getPressure(rho, u, gama)
    acc_g = libsx.getAcc_g_smth(pos, m, 1.0, eps)
    acc_sph = libsx.getAcc_sph(pos, v, rho, P, c, h, m, gama, 0.1, ALPHA, 2.0)
    acc_tot = f32(acc_g + acc_sph)
    acc_g, c, divV = f32(acc_g), f32(c), f32(divV)
    cols = [pos[:, 0], pos[:, 1], pos[:, 2], v[:, 0], v[:, 1], v[:, 2], acc_g[:, 0], acc_g[:, 1], acc_g[:, 2],
            acc_tot[:, 0], acc_tot[:, 1], acc_tot[:, 2], h, c, divV, eps]
    np.savez_compressed(IN_NPZ, pos=pos, vel=v, m=m, u=u, rho=rho, acc_g=acc_g, acc_tot=acc_tot, h=h, c=c,
                        divV=divV, eps=eps, c_cfl=C_CFL, alpha=ALPHA)
    os.makedirs(os.path.dirname(IN_BIN), exist_ok=True)
    with open(IN_BIN, "wb") as fh:
        np.array([n], dtype=np.int32).tofile(fh)
        np.array([C_CFL, ALPHA], dtype=np.float32).tofile(fh)
        np.concatenate([np.asarray(col, dtype=np.float32) for col in cols]).tofile(fh)
    print("wrote", IN_NPZ, IN_BIN)


def run(out_bin):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_timestep")
    subprocess.check_call([exe, IN_BIN, out_bin])


def merge(out_bin):
    d = dict(np.load(IN_NPZ))
    with open(out_bin, "rb") as fh:
        n = int(np.fromfile(fh, dtype=np.int32, count=1)[0])
        out = np.fromfile(fh, dtype=np.float32, count=4 * n).reshape(4, n)
    assert n == d["pos"].shape[0]
    d.update(dt=out[0], dhdt=out[1], abs_acc_g=out[2], abs_acc_tot=out[3])
    np.savez_compressed(OUT_NPZ, **d)
    print("wrote", OUT_NPZ)


if __name__ == "__main__":
    if len(sys.argv) < 3 or sys.argv[1] not in ("inputs", "run", "merge"):
        sys.exit(__doc__)
    {"inputs": inputs, "run": run, "merge": merge}[sys.argv[1]](sys.argv[2])
