"""Per-row cost of the reference's own CPU functions against the oracle's C
restatement, on the same rows of the same N = 1,048,576 Evrard state, one
core each.  The benchmark's CPU figures (`cpu_baseline` and `--impl
reference`) time the restatement because the reference's sources do not
travel to the GPU host; this script shows what that stand-in costs against
the reference's numba code where the reference is checked out.

    python tests/golden/time_reference.py /path/to/reference [rows]

For a contiguous row slice [nbeg, nend) -- the `_mpi` forms' own argument --
it times h_smooth_fast_mpi, getDensity_mpi, getAcc_g_smth_mpi,
getAcc_sph_mpi and get_dU_mpi (sph_code/libsx.py:52-86, 270-347, 498-564,
669-705, 854-902; numba-compiled before the clock starts) against the
oracle's h search, density, direct gravity and hydro rows with one OpenMP
thread, from the same untimed set-up (h of the rows brought into the
reference's 50 +- 5 window first, as the driver's loop starts each h search
from the previous step's h).  Prints one JSON line with seconds per row.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main(ref_root, nrows=24, n=1 << 20):
    sys.path.insert(0, os.path.join(ref_root, "sph_code"))
    sys.path.insert(0, ROOT)
    import libsx  # noqa: E402  (the reference)
    import oracle as oc  # noqa: E402
    from bench import cpu_state  # noqa: E402

    ic = cpu_state(n, n_ngb=50)
    pos, m, v, u = ic["pos"], ic["m"], ic["vel"], ic["u"]
    gama, eta, alpha, beta = 5.0 / 3.0, 0.1, 1.0, 2.0
    eps = np.full(n, 0.01)
    rho = ic["rho"]
    P = (gama - 1.0) * rho * u
    c = np.sqrt(gama * (gama - 1.0) * u)
    nbeg = n // 3
    nend = nbeg + nrows
    rows = np.arange(nbeg, nend)
    oc.build()
    h = ic["h"].copy()
    h[rows] = oc.h_smooth_rows(pos, h, rows, n_ngb=50, tol=5, max_iter=2000)[0]

    # compile the numba functions on a small problem (its own h, in the window)
    k = 256
    hk = oc.h_smooth_rows(pos[:k], np.full(k, 0.3), None, n_ngb=50, tol=5, max_iter=100000)[0]
    libsx.h_smooth_fast_mpi(0, 2, pos[:k], hk)
    libsx.getDensity_mpi(0, 2, pos[:k], m[:k], h[:k])
    libsx.getAcc_g_smth_mpi(0, 2, pos[:k], m[:k], 1.0, eps[:k])
    libsx.getAcc_sph_mpi(0, 2, pos[:k], v[:k], rho[:k], P[:k], c[:k], h[:k], m[:k], gama, eta, alpha, beta)
    libsx.get_dU_mpi(0, 2, pos[:k], v[:k], rho[:k], P[:k], c[:k], h[:k], m[:k], gama, eta, alpha, beta)

    ref = {}
    t0 = time.perf_counter()
    libsx.h_smooth_fast_mpi(nbeg, nend, pos, h)
    ref["h"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    libsx.getDensity_mpi(nbeg, nend, pos, m, h)
    ref["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    libsx.getAcc_g_smth_mpi(nbeg, nend, pos, m, 1.0, eps)
    ref["gravity"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    libsx.getAcc_sph_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
    ref["acc_sph"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    libsx.get_dU_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta)
    ref["dudt"] = time.perf_counter() - t0

    oc.set_threads(1)
    port = {}
    t0 = time.perf_counter()
    oc.h_smooth_rows(pos, h, rows, n_ngb=50, tol=5, max_iter=2000)
    port["h"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    oc.density_rows(pos, m, h, rows)
    port["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    oc.grav_direct_rows(pos, m, 1.0, eps, rows)
    port["gravity"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    oc.hydro_rows(pos, v, rho, P, c, h, m, 0, alpha, beta, eta, rows=rows, want_dudt=False)
    port["acc_sph"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    oc.hydro_rows(pos, v, rho, P, c, h, m, 0, alpha, beta, eta, rows=rows, want_acc=False)
    port["dudt"] = time.perf_counter() - t0

    per = lambda d: {k: d[k] / nrows for k in d}  # noqa: E731
    out = {"n": n, "rows": nrows, "cores": 1,
           "reference_s_per_row": per(ref), "port_s_per_row": per(port),
           "reference_total_s_per_row": sum(ref.values()) / nrows,
           "port_total_s_per_row": sum(port.values()) / nrows}
    out["reference_over_port"] = out["reference_total_s_per_row"] / out["port_total_s_per_row"]
    print(json.dumps(out))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(__doc__)
    main(sys.argv[1], *(int(a) for a in sys.argv[2:3]))
