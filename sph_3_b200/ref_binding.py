"""ctypes binding of libsph3 for the reference's own sph_code/ directory.

A maintainer who wants the reference drivers to call the GPU path without
this package's Python layer copies this file next to sph_code/libsx.py and
imports these functions in place of the numba ones.  It replaces
getDensity (sph_code/libsx.py:10-47) and getAcc_g_smth (sph_code/libsx.py:
623-652) with the same signatures and FP64 results; the other functions
follow the same pattern with the SPH3_DO_* flags of include/sph3.h.
Only ctypes and NumPy are needed.
"""
import ctypes
import os

import numpy as np

lib = ctypes.CDLL(os.environ.get("SPH3_LIB", os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                                                          "libsph3.so")))
P, I32, I64, F64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double


class Config(ctypes.Structure):           # mirrors sph3_config in include/sph3.h
    _fields_ = [(n, t) for n, t in [
        ("precision", I32), ("h_mode", I32), ("visc", I32), ("step_order", I32),
        ("n_ngb", I32), ("n_ngb_tol", I32), ("h_max_iter", I32), ("n_boot", I32),
        ("leaf_size", I32), ("stack_cap", I32), ("max_level", I32), ("gravity", I32),
        ("quadrupole", I32), ("use_graph", I32), ("timing", I32), ("walk_warps", I32),
        ("list_cap", I32), ("mac", I32), ("eps_from_h", I32), ("step_potential", I32),
        ("gamma", F64), ("alpha", F64), ("beta", F64), ("eta", F64), ("G", F64), ("theta", F64), ("eps", F64), ("box", F64 * 3),
        ("reserved_d", F64 * 4)]]


lib.sph3_default_config.argtypes = [P]
lib.sph3_ctx_create.argtypes = [P, ctypes.c_int, P]
lib.sph3_set_particles.argtypes = [P, I64, P, P, P, P, P, P, ctypes.c_int, P]
lib.sph3_set_field.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P]
lib.sph3_compute.argtypes = [P, ctypes.c_uint32, P]
lib.sph3_get_field.argtypes = [P, ctypes.c_int, P, I64, I64, ctypes.c_int, P]
lib.sph3_ctx_destroy.argtypes = [P]
lib.sph3_gravity_pairsum.argtypes = [P, ctypes.c_int, I64, I64, P, ctypes.c_int, P]
SPH3_DO_DENSITY, SPH3_GSUM_ROWS = 0x8, 0
SPH3_FIELD_RHO, SPH3_FIELD_ACC_G = 6, 12


def _ctx(**over):
    cfg = Config(); lib.sph3_default_config(ctypes.byref(cfg))
    cfg.precision = 1; cfg.h_mode = 1                 # FP64, the reference's h rule
    for k, v in over.items(): setattr(cfg, k, v)
    ctx = P(); rc = lib.sph3_ctx_create(ctypes.byref(cfg), 0, ctypes.byref(ctx))   # device 0
    if rc: raise RuntimeError("sph3_ctx_create: %d" % rc)
    return ctx


def _ptr(a): return a.ctypes.data_as(P)


def getDensity(pos, m, h):
    pos = np.ascontiguousarray(pos, np.float64); n = len(m)
    m = np.ascontiguousarray(m, np.float64); h = np.ascontiguousarray(h, np.float64)
    ctx = _ctx(gravity=0)
    try:
        zeros = np.zeros((n, 3)); u = np.zeros(n)
        for rc in (lib.sph3_set_particles(ctx, n, _ptr(pos), _ptr(zeros), _ptr(m), _ptr(u), _ptr(h), None, 0, None),
                   lib.sph3_compute(ctx, SPH3_DO_DENSITY, None)):
            if rc: raise RuntimeError("sph3: %d" % rc)
        rho = np.empty(n)
        rc = lib.sph3_get_field(ctx, SPH3_FIELD_RHO, _ptr(rho), 0, n, 0, None)
        if rc: raise RuntimeError("sph3_get_field: %d" % rc)
        return rho
    finally:
        lib.sph3_ctx_destroy(ctx)


def getAcc_g_smth(pos, mass, G, epsilon):
    pos = np.ascontiguousarray(pos, np.float64); n = len(mass)
    mass = np.ascontiguousarray(mass, np.float64)
    eps = np.full(n, float(epsilon)) if np.ndim(epsilon) == 0 else np.ascontiguousarray(epsilon, np.float64)
    ctx = _ctx(G=float(G))
    try:
        z3 = np.zeros((n, 3)); z1 = np.zeros(n); acc = np.empty((n, 3))
        # the reference's direct sum in its own summation order (bit for bit)
        for rc in (lib.sph3_set_particles(ctx, n, _ptr(pos), _ptr(z3), _ptr(mass), _ptr(z1), _ptr(z1), _ptr(eps), 0, None),
                   lib.sph3_gravity_pairsum(ctx, SPH3_GSUM_ROWS, 0, n, _ptr(acc), 0, None)):
            if rc: raise RuntimeError("sph3: %d" % rc)
        return acc
    finally:
        lib.sph3_ctx_destroy(ctx)
