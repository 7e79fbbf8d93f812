"""Writes tests/golden/ppm_evrard.npz from the reference's 1-D PPM Evrard
solution (sph_code/ppm_profile/ppm1oaf, 350 radial zones), converted to the
code units of the Evrard test (M = R = G = 1) the way the reference's plot
script does (Particles_in_BH_Tree_III/Evrard_Collapse_2024/pplot3.py:12-49):
radius / 1.257607e11, density / (3 / 4 pi) then * (3 / 4 pi), radial velocity
/ sqrt(e*) * 1e-8, pressure / (rho* e*) * 1e-16 then * (3 / 4 pi), with
e* = 1.054811e-1 / 1.05.  Run with the reference's checkout as the argument
(or in the SPH3_REFERENCE environment variable):

    python tests/golden/make_ppm.py /path/to/reference

The fixture is what the tests read.
"""
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ppm_evrard.npz")


def main(ref_root):
    src = os.path.join(ref_root, "sph_code", "ppm_profile", "ppm1oaf")
    rost = 3.0 / 4.0 / np.pi
    est = 1.054811e-1 / 1.05
    pst = rost * est
    vst = np.sqrt(est)
    rst = 1.257607
    with open(src) as fh:
        lines = [ln.split() for ln in fh if ln.strip()]
    t_phys = float(lines[0][1])
    rows = np.array([[float(v) for v in ln[1:5]] for ln in lines[1:351]])
    radius = rows[:, 0] / rst * 1e-11
    rho = rows[:, 1] / rost * (3.0 / (4 * np.pi))
    press = rows[:, 2] / pst * 1e-16 * (3.0 / (4 * np.pi))
    vr = rows[:, 3] / vst * 1e-8
    np.savez(OUT, radius=radius, rho=rho, press=press, vr=vr, t_header=t_phys)
    print(OUT, radius.min(), radius.max(), rho.max())


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPH3_REFERENCE")
    if not root:
        sys.exit("usage: make_ppm.py REFERENCE_ROOT  (or set SPH3_REFERENCE)")
    main(root)
