"""Generate the golden vectors in this folder by running the reference's own
numba functions (sph_code/libsx.py, sph_code/shear.py) on seeded inputs.

Run once, in a container that has the reference checked out:

    python tests/golden/make_golden.py /path/to/reference [set ...]

(or with the path in the SPH3_REFERENCE environment variable); sets are
``hydro`` (evrard600, evrard1500 and the edge cases) and ``gravity``
(grav_forms), all of them by default.  The output ``*.npz`` files are
committed; tests read only them.  Inputs are the Evrard-profile initial
conditions used throughout the tests (r = R sqrt(U), isotropic directions,
equal masses) at small N, plus edge cases.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def evrard(n, seed, R=1.0, M=1.0):
    rng = np.random.default_rng(seed)
    u = rng.random(n)
    r = R * np.sqrt(u)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pos = d * r[:, None]
    m = np.full(n, M / n)
    return pos, m


def gravity_forms(libsx):
    """Every gravity form of the reference on one unequal-mass, unequal-eps
    set: the symmetric full field, its x twin, a row slice, the mimj partial
    arrays of a three-way row partition, getPE, and do_smoothingX with query
    points distinct from the particles (some outside the cloud, one on a
    particle)."""
    n = 700
    pos, _ = evrard(n, 21)
    rng = np.random.default_rng(2100)
    m = (0.5 + rng.random(n)) / n
    eps = 0.005 + 0.015 * rng.random(n)
    G = 1.0
    acc_sym = libsx.getAcc_g_smth(pos, m, G, eps)
    acc_x = libsx.getAcc_g_smthx(pos, m, G, eps)
    acc_rows = libsx.getAcc_g_smth_mpi(150, 420, pos, m, G, eps)
    parts = np.array([[0, 230], [230, 520], [520, n]])
    mimj = np.stack([libsx.getAcc_g_smth_mimj_mpi(int(b), int(e), pos, m, G, eps) for b, e in parts])
    PE = libsx.getPE(pos, m, G, eps)
    q = np.concatenate([rng.normal(scale=0.6, size=(120, 3)), 1.5 * rng.normal(size=(29, 3)), pos[[17]]])
    hq = libsx.do_smoothingX((pos, q))
    np.savez_compressed(os.path.join(HERE, "grav_forms.npz"), pos=pos, m=m, eps=eps, G=G,
                        acc_sym=acc_sym, acc_x=acc_x, acc_rows=acc_rows, acc_rows_range=np.array([150, 420]),
                        mimj=mimj, mimj_parts=parts, PE=PE, q=q, hq=hq)
    print("wrote grav_forms", n)


def main(ref_root, sets=("hydro", "gravity")):
    sys.path.insert(0, os.path.join(ref_root, "sph_code"))
    import libsx  # noqa: E402  (the reference)
    import shear  # noqa: E402  (the reference)

    if "gravity" in sets:
        gravity_forms(libsx)
    if "hydro" not in sets:
        return
    gama, alpha, beta, eta, G = 5.0 / 3.0, 1.0, 2.0, 0.1, 1.0
    cases = {"evrard600": (600, 7), "evrard1500": (1500, 11)}
    for name, (n, seed) in cases.items():
        pos, m = evrard(n, seed)
        rng = np.random.default_rng(seed + 1000)
        v = rng.normal(scale=0.1, size=(n, 3))
        u = 0.05 * (1.0 + 0.5 * rng.random(n))
        eps = np.full(n, 0.01)
        h0 = libsx.smoothing_length_mpi(0, n, pos)
        h = libsx.h_smooth_fast(pos, h0)
        rho = libsx.getDensity(pos, m, h)
        P = libsx.getPressure(rho, u, gama)
        c = np.sqrt(gama * (gama - 1.0) * u)
        acc_sph = libsx.getAcc_sph(pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
        dudt = libsx.get_dU(pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
        acc_mg = libsx.getAcc_sph_mpiXXX(0, n, pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
        dudt_mg = libsx.get_dU_mpiXXXX(0, n, pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
        divV, curlV = shear.div_curlVel(pos, v, rho, m, h)
        acc_sh = shear.getAcc_sph_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha)
        dudt_sh = shear.get_dU_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha)
        acc_g = libsx.getAcc_g_smth_mpi(0, n, pos, m, G, eps)
        acc_g_sym = libsx.getAcc_g_smth(pos, m, G, eps)
        KE = libsx.getKE(v, m)
        PE = libsx.getPE(pos, m, G, eps)
        # the h search from a perturbed start, and the row-slice variants
        h_pert = h0 * (1.0 + 0.2 * (rng.random(n) - 0.5))
        h_from_pert = libsx.h_smooth_fast_mpi(n // 3, n // 3 + 100, pos, h_pert)
        rho_mpi = libsx.getDensity_mpi(n // 4, n // 4 + 50, pos, m, h)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            pos=pos, vel=v, m=m, u=u, eps=eps, h0=h0, h=h, rho=rho, P=P, c=c,
            acc_sph=acc_sph, dudt=dudt, acc_mg=acc_mg, dudt_mg=dudt_mg, divV=divV,
            curlV=curlV, acc_sh=acc_sh, dudt_sh=dudt_sh, acc_g=acc_g, acc_g_sym=acc_g_sym,
            KE=KE, PE=PE, h_pert=h_pert, h_from_pert=h_from_pert,
            h_from_pert_range=np.array([n // 3, n // 3 + 100]), rho_mpi=rho_mpi,
            rho_mpi_range=np.array([n // 4, n // 4 + 50]),
            consts=np.array([gama, alpha, beta, eta, G]))
        print("wrote", name, n)

    # edge cases: a coincident pair (gravity skipped: the reference divides by
    # zero there), a particle count of 1, and a tiny isolated clump
    n = 120
    pos, m = evrard(n, 3)
    pos[5] = pos[4]
    v = np.zeros((n, 3)); u = np.full(n, 0.05)
    h = libsx.smoothing_length_mpi(0, n, pos)
    rho = libsx.getDensity(pos, m, h)
    P = libsx.getPressure(rho, u, gama)
    c = np.sqrt(gama * (gama - 1.0) * u)
    acc_sph = libsx.getAcc_sph(pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
    dudt = libsx.get_dU(pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
    np.savez_compressed(os.path.join(HERE, "coincident120.npz"), pos=pos, vel=v, m=m, u=u, h=h,
                        rho=rho, P=P, c=c, acc_sph=acc_sph, dudt=dudt,
                        consts=np.array([gama, alpha, beta, eta, G]))
    pos1 = np.array([[0.1, -0.2, 0.3]]); m1 = np.array([0.5]); h1 = np.array([0.05])
    rho1 = libsx.getDensity(pos1, m1, h1)
    np.savez_compressed(os.path.join(HERE, "single.npz"), pos=pos1, m=m1, h=h1, rho=rho1)
    print("wrote edge cases")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPH3_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [hydro] [gravity]  (or set SPH3_REFERENCE)")
    main(root, tuple(sys.argv[2:]) or ("hydro", "gravity"))
