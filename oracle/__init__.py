"""CPU oracle for the SPH_3 per-step particle path -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.  The product (``sph_3_b200``) never does.

``sph_oracle.c`` restates the reference's numba functions in C (see its
header); this module builds it with gcc and exposes NumPy wrappers whose names
and signatures follow the reference:

=====================================  ==========================================
wrapper                                reference (sph_code/...)
=====================================  ==========================================
getDensity / getDensity_mpi            libsx.py:10-44 / 50-86
h_smooth_fast / h_smooth_fast_mpi      libsx.py:804-845 / 852-902
smoothing_length_mpi / do_smoothingX   libsx.py:779-800 / 752-774
getAcc_sph / getAcc_sph_mpi            libsx.py:100-177 / 268-347
getAcc_sph_mpiXXX                      libsx.py:183-262
get_dU / get_dU_mpi / get_dU_mpiXXXX   libsx.py:353-421 / 496-564 / 427-491
getAcc_g_smth_mpi / getAcc_g_smthx     libsx.py:667-705 / 710-747
getAcc_g_smth                          libsx.py:623-662 (pairwise-symmetric order)
getKE / getPE                          libsx.py:569-579 / 583-620
div_curlVel / div_curlVel_mpi          shear.py:7-69 / 76-142
getAcc_sph_shear / get_dU_shear (+mpi) shear.py:149-326 / 332-485
=====================================  ==========================================

Extensions used by the tests (all reduce to the reference at their defaults):
``n_ngb``/``tol``/``max_iter`` for the h search, ``box`` for a periodic
minimum image, and ``rows`` index lists for sampled-row checks at large N.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "sph_oracle.c")
_BUILD = os.path.join(_HERE, "_build")
_LIB_PATH = os.path.join(_BUILD, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc, OpenMP, no FP contraction)."""
    os.makedirs(_BUILD, exist_ok=True)
    if (not force and os.path.exists(_LIB_PATH)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(_SRC)):
        return _LIB_PATH
    tmp = _LIB_PATH + ".tmp%d" % os.getpid()
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
           "-shared", "-o", tmp, _SRC, "-lm"]
    subprocess.check_call(cmd)
    os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


def build_ref(ref_root=None):
    """Compile oracle/_ref/ref_timestep and oracle/_ref/ref_cooling (the
    reference's own GPU time-step and heating/cooling kernels behind small
    drivers, oracle/build_ref.sh) where the reference is checked out; returns
    the binaries' paths, or None when it is not."""
    cmd = ["sh", os.path.join(_HERE, "build_ref.sh")] + ([ref_root] if ref_root else [])
    r = subprocess.run(cmd, capture_output=True, text=True)
    return r.stdout.split() if r.returncode == 0 else None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    I = ctypes.c_int64
    D = ctypes.c_double
    C = ctypes.c_int
    sigs = {
        "orc_density": [I, P, P, P, P, I, P, P],
        "orc_neighbours": [I, P, P, I, P, P, I],
        "orc_h_smooth": [I, P, P, P, I, C, C, I, P, P, P],
        "orc_count_within": [I, P, P, P, I, P, P],
        "orc_smoothing_length": [I, P, P, I, C, P, P],
        "orc_div_curl": [I, P, P, P, P, P, P, I, P, P, P],
        "orc_hydro": [I, P, P, P, P, P, P, P, P, P, C, D, D, D, P, I, P, P, P],
        "orc_grav_direct": [I, P, P, D, P, P, I, P, P],
        "orc_grav_sym": [I, P, P, D, P, P],
        "orc_grav_mimj": [I, P, P, D, P, I, I, P],
        "orc_smoothing_points": [I, P, I, P, C, P],
        "orc_pe": [I, P, P, D, P],
        "orc_ke": [I, P, P],
        "orc_timestep": [I, P, P, P, P, P, P, P, P, D, D, C, P, I, P, P],
        "orc_hcooling": [I, P, P, P, P, P, P, P, ctypes.c_float, P, P, P, P, P, P, P, P, ctypes.c_int32],
        "orc_set_threads": [C],
        "orc_num_threads": [],
    }
    for name, args in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
    lib.orc_neighbours.restype = ctypes.c_int64
    lib.orc_pe.restype = ctypes.c_double
    lib.orc_ke.restype = ctypes.c_double
    lib.orc_num_threads.restype = ctypes.c_int
    lib.orc_set_threads.restype = None
    _lib = lib
    return lib


def set_threads(n: int) -> None:
    _load().orc_set_threads(int(n))


def num_threads() -> int:
    return int(_load().orc_num_threads())


# ---------------------------------------------------------------- helpers
def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _rows(n, rows, nbeg=None, nend=None):
    if rows is None:
        if nbeg is None:
            nbeg, nend = 0, n
        rows = np.arange(nbeg, nend, dtype=np.int64)
    return np.ascontiguousarray(rows, dtype=np.int64)


def _box(box):
    if box is None:
        return None
    b = np.zeros(3, dtype=np.float64)
    b[:] = box
    return b


# ---------------------------------------------------------------- density / h
def density_rows(pos, m, h, rows=None, box=None):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]
    m = _f64(m); h = _f64(h); r = _rows(n, rows); b = _box(box)
    out = np.zeros(r.shape[0])
    _load().orc_density(n, _ptr(pos), _ptr(m), _ptr(h), _ptr(r), r.shape[0], _ptr(b), _ptr(out))
    return out


def getDensity(pos, m, h):
    return density_rows(pos, m, h)


def getDensity_mpi(nbeg, nend, pos, m, h):
    n = _f64(pos, (-1, 3)).shape[0]
    return density_rows(pos, m, h, _rows(n, None, nbeg, nend))


def neighbours(pos, h, i, box=None):
    """Sorted indices j with |r_ij| <= 2 * (h_i + h_j) / 2 for particle i."""
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; h = _f64(h); b = _box(box)
    cap = 4096
    while True:
        out = np.empty(cap, dtype=np.int64)
        k = _load().orc_neighbours(n, _ptr(pos), _ptr(h), int(i), _ptr(b), _ptr(out), cap)
        if k <= cap:
            return out[:k].copy()
        cap = int(k)


def h_smooth_rows(pos, h, rows=None, n_ngb=50, tol=5, max_iter=1 << 40, box=None):
    """Returns (h, steps) for the rows; steps = -1 where max_iter was hit."""
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; h = _f64(h)
    r = _rows(n, rows); b = _box(box)
    out = np.zeros(r.shape[0]); st = np.zeros(r.shape[0], dtype=np.int64)
    _load().orc_h_smooth(n, _ptr(pos), _ptr(h), _ptr(r), r.shape[0], int(n_ngb), int(tol),
                         int(max_iter), _ptr(b), _ptr(out), _ptr(st))
    return out, st


def h_smooth_fast(pos, h):
    return h_smooth_rows(pos, h)[0]


def h_smooth_fast_mpi(nbeg, nend, pos, h):
    n = _f64(pos, (-1, 3)).shape[0]
    return h_smooth_rows(pos, h, _rows(n, None, nbeg, nend))[0]


def count_within(pos, h, rows=None, box=None):
    """N(dist < 2 h_i) for each row (the h search's own count)."""
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; h = _f64(h); r = _rows(n, rows); b = _box(box)
    out = np.zeros(r.shape[0], dtype=np.int64)
    _load().orc_count_within(n, _ptr(pos), _ptr(h), _ptr(r), r.shape[0], _ptr(b), _ptr(out))
    return out


def smoothing_length_rows(pos, rows=None, k=50, box=None):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; r = _rows(n, rows); b = _box(box)
    out = np.zeros(r.shape[0])
    _load().orc_smoothing_length(n, _ptr(pos), _ptr(r), r.shape[0], int(k), _ptr(b), _ptr(out))
    return out


def smoothing_length_mpi(nbeg, nend, pos):
    n = _f64(pos, (-1, 3)).shape[0]
    return smoothing_length_rows(pos, _rows(n, None, nbeg, nend))


def do_smoothingX(poz):
    """h = half the distance from each subpos row to its 51st-nearest pos row."""
    pos, subpos = poz
    pos = _f64(pos, (-1, 3))
    subpos = _f64(subpos, (-1, 3))
    if subpos.shape == pos.shape and np.array_equal(subpos, pos):
        return smoothing_length_rows(pos)
    return smoothing_points(pos, subpos)


def smoothing_points(pos, q, k=50):
    """0.5 x the k-th (0-based) smallest distance from each row of q to the rows of pos."""
    pos = _f64(pos, (-1, 3))
    q = _f64(q, (-1, 3))
    out = np.zeros(q.shape[0])
    _load().orc_smoothing_points(pos.shape[0], _ptr(pos), q.shape[0], _ptr(q), int(k), _ptr(out))
    return out


def getPressure(rho, u, gama):
    return (gama - 1.0) * rho * u


# ---------------------------------------------------------------- div/curl, hydro
def div_curl_rows(pos, v, rho, m, h, rows=None, box=None):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; v = _f64(v, (-1, 3))
    rho = _f64(rho); m = _f64(m); h = _f64(h); r = _rows(n, rows); b = _box(box)
    dv = np.zeros(r.shape[0]); cv = np.zeros(r.shape[0])
    _load().orc_div_curl(n, _ptr(pos), _ptr(v), _ptr(rho), _ptr(m), _ptr(h), _ptr(r),
                         r.shape[0], _ptr(b), _ptr(dv), _ptr(cv))
    return dv, cv


def div_curlVel(pos, v, rho, m, h):
    return div_curl_rows(pos, v, rho, m, h)


def div_curlVel_mpi(nbeg, nend, pos, v, rho, m, h):
    n = _f64(pos, (-1, 3)).shape[0]
    return div_curl_rows(pos, v, rho, m, h, _rows(n, None, nbeg, nend))


VISC_SIGNAL, VISC_MG83, VISC_BALSARA = 0, 1, 2


def hydro_rows(pos, v, rho, P, c, h, m, visc=VISC_SIGNAL, alpha=1.0, beta=2.0, eta=0.1,
               divV=None, curlV=None, rows=None, box=None, want_acc=True, want_dudt=True):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; v = _f64(v, (-1, 3))
    rho = _f64(rho); P = _f64(P); c = _f64(c); h = _f64(h); m = _f64(m)
    dv = _f64(divV) if divV is not None else None
    cv = _f64(curlV) if curlV is not None else None
    if visc == VISC_BALSARA and (dv is None or cv is None):
        raise ValueError("Balsara viscosity needs divV and curlV")
    r = _rows(n, rows); b = _box(box)
    acc = np.zeros((r.shape[0], 3)) if want_acc else None
    du = np.zeros(r.shape[0]) if want_dudt else None
    _load().orc_hydro(n, _ptr(pos), _ptr(v), _ptr(rho), _ptr(P), _ptr(c), _ptr(h), _ptr(m),
                      _ptr(dv), _ptr(cv), int(visc), float(alpha), float(beta), float(eta),
                      _ptr(r), r.shape[0], _ptr(b), _ptr(acc), _ptr(du))
    return acc, du


def getAcc_sph(pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_SIGNAL, alpha, beta, eta, want_dudt=False)[0]


def getAcc_sph_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    n = _f64(pos, (-1, 3)).shape[0]
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_SIGNAL, alpha, beta, eta,
                      rows=_rows(n, None, nbeg, nend), want_dudt=False)[0]


def getAcc_sph_mpiXXX(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    n = _f64(pos, (-1, 3)).shape[0]
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_MG83, alpha, beta, eta,
                      rows=_rows(n, None, nbeg, nend), want_dudt=False)[0]


def get_dU(pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_SIGNAL, alpha, beta, eta, want_acc=False)[1]


def get_dU_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    n = _f64(pos, (-1, 3)).shape[0]
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_SIGNAL, alpha, beta, eta,
                      rows=_rows(n, None, nbeg, nend), want_acc=False)[1]


def get_dU_mpiXXXX(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    n = _f64(pos, (-1, 3)).shape[0]
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_MG83, alpha, beta, eta,
                      rows=_rows(n, None, nbeg, nend), want_acc=False)[1]


def getAcc_sph_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha):
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_BALSARA, alpha, 0.0, 0.0, divV, curlV,
                      want_dudt=False)[0]


def getAcc_sph_shear_mpi(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha):
    n = _f64(pos, (-1, 3)).shape[0]
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_BALSARA, alpha, 0.0, 0.0, divV, curlV,
                      rows=_rows(n, None, nbeg, nend), want_dudt=False)[0]


def get_dU_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha):
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_BALSARA, alpha, 0.0, 0.0, divV, curlV,
                      want_acc=False)[1]


def get_dU_shear_mpi(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha):
    n = _f64(pos, (-1, 3)).shape[0]
    return hydro_rows(pos, v, rho, P, c, h, m, VISC_BALSARA, alpha, 0.0, 0.0, divV, curlV,
                      rows=_rows(n, None, nbeg, nend), want_acc=False)[1]


# ---------------------------------------------------------------- gravity / energy
def grav_direct_rows(pos, mass, G, eps, rows=None, want_phi=False):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; mass = _f64(mass)
    eps = np.broadcast_to(_f64(eps), (n,)).copy() if np.ndim(eps) == 0 else _f64(eps)
    r = _rows(n, rows)
    acc = np.zeros((r.shape[0], 3))
    phi = np.zeros(r.shape[0]) if want_phi else None
    _load().orc_grav_direct(n, _ptr(pos), _ptr(mass), float(G), _ptr(eps), _ptr(r), r.shape[0],
                            _ptr(acc), _ptr(phi))
    return (acc, phi) if want_phi else acc


def getAcc_g_smth_mpi(nbeg, nend, pos, mass, G, epsilon):
    n = _f64(pos, (-1, 3)).shape[0]
    return grav_direct_rows(pos, mass, G, epsilon, _rows(n, None, nbeg, nend))


def getAcc_g_smthx(pos, mass, G, epsilon):
    return grav_direct_rows(pos, mass, G, epsilon)


def getAcc_g_smth(pos, mass, G, epsilon):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; mass = _f64(mass)
    eps = np.broadcast_to(_f64(epsilon), (n,)).copy() if np.ndim(epsilon) == 0 else _f64(epsilon)
    out = np.zeros((n, 3))
    _load().orc_grav_sym(n, _ptr(pos), _ptr(mass), float(G), _ptr(eps), _ptr(out))
    return out


def getAcc_g_smth_mimj_mpi(nbeg, nend, pos, mass, G, epsilon):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]; mass = _f64(mass)
    eps = np.broadcast_to(_f64(epsilon), (n,)).copy() if np.ndim(epsilon) == 0 else _f64(epsilon)
    out = np.zeros((n, 3))
    _load().orc_grav_mimj(n, _ptr(pos), _ptr(mass), float(G), _ptr(eps), int(nbeg), int(nend), _ptr(out))
    return out


def getPE(pos, m, G, epsilon):
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]
    eps = np.broadcast_to(_f64(epsilon), (n,)).copy() if np.ndim(epsilon) == 0 else _f64(epsilon)
    return float(_load().orc_pe(n, _ptr(pos), _ptr(_f64(m)), float(G), _ptr(eps)))


def getKE(v, m):
    v = _f64(v, (-1, 3))
    return float(_load().orc_ke(v.shape[0], _ptr(v), _ptr(_f64(m))))


from .step import serial_first_step, serial_step  # noqa: E402,F401

def timestep_rows(pos, v, acc_tot, acc_g, h, c, divV, eps, c_cfl, alpha, neighbours=False, rows=None):
    """Per-particle dt and dh/dt of dt_array_indiv_dt (see orc_timestep)."""
    pos = _f64(pos, (-1, 3)); n = pos.shape[0]
    v = _f64(v, (-1, 3)); at = _f64(acc_tot, (-1, 3)); ag = _f64(acc_g, (-1, 3))
    h = _f64(h); c = _f64(c); dv = _f64(divV)
    eps = np.broadcast_to(_f64(eps), (n,)).copy() if np.ndim(eps) == 0 else _f64(eps)
    r = _rows(n, rows)
    dt = np.zeros(r.shape[0]); dh = np.zeros(r.shape[0])
    _load().orc_timestep(n, _ptr(pos), _ptr(v), _ptr(at), _ptr(ag), _ptr(h), _ptr(c), _ptr(dv), _ptr(eps),
                         float(c_cfl), float(alpha), 1 if neighbours else 0, _ptr(r), r.shape[0], _ptr(dt), _ptr(dh))
    return dt, dh


def hcooling(table, units, dt, u, rho, pos, typ=None, z_index=1, ionfrac=True):
    """hcoolingZ restated in FP32 (orc_hcooling): returns (u_new, ionfrac or
    None).  `table` holds the arrays of the reference's cooling-table file
    (dims, kpc, nH, t, uEvol, metalz, uArr); `units` = (unit density cgs,
    unit time s, unit u cgs, unit length cm, kpc cm)."""
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    pos = f32(pos).reshape(-1, 3)
    n = pos.shape[0]
    x, y, z = f32(pos[:, 0]), f32(pos[:, 1]), f32(pos[:, 2])
    un = f32(u).copy()
    rh = f32(rho)
    dims = np.ascontiguousarray(table["dims"], dtype=np.int32)
    arrs = [f32(table[k]) for k in ("kpc", "nH", "t", "uEvol", "metalz", "uArr")]
    uv = f32(units)
    ty = None if typ is None else np.ascontiguousarray(typ, dtype=np.int32)
    ion = np.zeros((n, int(dims[4])), np.float32) if ionfrac else None
    vp = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _load().orc_hcooling(n, vp(ty), vp(un), vp(rh), vp(x), vp(y), vp(z), vp(ion), float(dt), vp(dims),
                         *[vp(a) for a in arrs], vp(uv), int(z_index))
    return un, ion
