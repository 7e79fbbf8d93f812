"""ctypes binding of the C ABI in include/sph3.h (sph_3_b200/lib/libsph3.so).

The library is built in-tree by ``python -m sph_3_b200.build`` (or
``__graft_entry__.build()``).  There is no fallback: if the library is missing
or cannot be loaded, every call raises :class:`LibraryError`.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
# SPH3_LIB selects another build of the library (e.g. side-by-side variants)
LIB_PATH = os.environ.get("SPH3_LIB") or os.path.join(HERE, "lib", "libsph3.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "sph3.h")


class LibraryError(RuntimeError):
    pass


class Sph3Error(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__("sph3 error %d (%s)%s" % (code, error_string(code), (": " + what) if what else ""))


def _consts():
    """#define constants of the header, parsed once (single source of truth)."""
    out = {}
    with open(HEADER) as fh:
        for line in fh:
            m = re.match(r"#define\s+(SPH3_\w+)\s+(0x[0-9a-fA-F]+|\d+)u?\b", line)
            if m:
                out[m.group(1)] = int(m.group(2), 0)
    return out


C = _consts()


class Config(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int32),
        ("h_mode", ctypes.c_int32),
        ("visc", ctypes.c_int32),
        ("step_order", ctypes.c_int32),
        ("n_ngb", ctypes.c_int32),
        ("n_ngb_tol", ctypes.c_int32),
        ("h_max_iter", ctypes.c_int32),
        ("n_boot", ctypes.c_int32),
        ("leaf_size", ctypes.c_int32),
        ("stack_cap", ctypes.c_int32),
        ("max_level", ctypes.c_int32),
        ("gravity", ctypes.c_int32),
        ("quadrupole", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("timing", ctypes.c_int32),
        ("walk_warps", ctypes.c_int32),
        ("list_cap", ctypes.c_int32),
        ("mac", ctypes.c_int32),
        ("eps_from_h", ctypes.c_int32),
        ("step_potential", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("beta", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("G", ctypes.c_double),
        ("theta", ctypes.c_double),
        ("eps", ctypes.c_double),
        ("box", ctypes.c_double * 3),
        ("reserved_d", ctypes.c_double * 4),
    ]


class CoolUnits(ctypes.Structure):
    _fields_ = [
        ("unit_density_cgs", ctypes.c_float),
        ("unit_time_s", ctypes.c_float),
        ("unit_u_cgs", ctypes.c_float),
        ("unit_length_cm", ctypes.c_float),
        ("kpc_cm", ctypes.c_float),
        ("z_index", ctypes.c_int32),
    ]


# every exported function with its ctypes signature
P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int32
U32 = ctypes.c_uint32
D = ctypes.c_double
SIGNATURES = {
    "sph3_version": (ctypes.c_int, []),
    "sph3_default_config": (None, [P]),
    "sph3_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "sph3_ctx_create": (ctypes.c_int, [P, ctypes.c_int, P]),
    "sph3_ctx_destroy": (ctypes.c_int, [P]),
    "sph3_set_config": (ctypes.c_int, [P, P]),
    "sph3_get_config": (ctypes.c_int, [P, P]),
    "sph3_set_clouds": (ctypes.c_int, [P, P, I32]),
    "sph3_set_particles": (ctypes.c_int, [P, I64, P, P, P, P, P, P, ctypes.c_int, P]),
    "sph3_num_particles": (I64, [P]),
    "sph3_set_field": (ctypes.c_int, [P, ctypes.c_int, P, ctypes.c_int, P]),
    "sph3_get_field": (ctypes.c_int, [P, ctypes.c_int, P, I64, I64, ctypes.c_int, P]),
    "sph3_compute": (ctypes.c_int, [P, U32, P]),
    "sph3_compute_rows": (ctypes.c_int, [P, U32, I64, I64, P]),
    "sph3_first_step": (ctypes.c_int, [P, D, P]),
    "sph3_step": (ctypes.c_int, [P, D, I32, P]),
    "sph3_energy": (ctypes.c_int, [P, P, P]),
    "sph3_status": (ctypes.c_int, [P, P, ctypes.c_int]),
    "sph3_gravity_direct_rows": (ctypes.c_int, [P, P, I64, P, P]),
    "sph3_neighbours": (ctypes.c_int, [P, P, I64, P, P, I64]),
    "sph3_pair_lists": (ctypes.c_int, [P, P, I64, P, P, I64]),
    "sph3_morton_order": (ctypes.c_int, [P, P, P]),
    "sph3_counters": (ctypes.c_int, [P, P, ctypes.c_int]),
    "sph3_phase_times": (ctypes.c_int, [P, P, ctypes.c_int]),
    "sph3_kernels_per_step": (ctypes.c_int, [P, P]),
    "sph3_probe_fp32_rate": (ctypes.c_int, [ctypes.c_int, P, P]),
    "sph3_timestep": (ctypes.c_int, [P, ctypes.c_double, ctypes.c_int, P, P]),
    "sph3_morton_sort_noalloc": (ctypes.c_int, [P, I64, I32, P, P, P, P]),
    "sph3_gravity_pairsum": (ctypes.c_int, [P, ctypes.c_int, I64, I64, P, ctypes.c_int, P]),
    "sph3_potential_pairsum": (ctypes.c_int, [P, P, P]),
    "sph3_kth_distance": (ctypes.c_int, [P, P, I64, I32, P, ctypes.c_int, P]),
    "sph3_step_io": (ctypes.c_int, [P, D, I32, I32, P, P, I32, P, P, P]),
    "sph3_cool_table_create": (ctypes.c_int, [ctypes.c_int, P, P, P, P, P, P, P, P]),
    "sph3_cool_table_destroy": (ctypes.c_int, [P]),
    "sph3_cool_table_dims": (ctypes.c_int, [P, P, P]),
    "sph3_hcooling": (ctypes.c_int, [P, P, ctypes.c_float, I64, P, P, P, P, P, P, P, P, P]),
    "sph3_set_cooling": (ctypes.c_int, [P, P, P]),
    "sph3_cool_now": (ctypes.c_int, [P, D, P]),
    "sph3_get_ionfrac": (ctypes.c_int, [P, P, I64]),
}

_lib = None


def load():
    """Loads libsph3.so (raises LibraryError if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryError("libsph3.so is not built (%s); run `python -m sph_3_b200.build`" % LIB_PATH)
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise LibraryError("cannot load %s: %s" % (LIB_PATH, e)) from e
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def error_string(code):
    try:
        return load().sph3_error_string(int(code)).decode()
    except LibraryError:
        return "library not loaded"


def check(code, what=""):
    if code != 0:
        raise Sph3Error(code, what)


def default_config() -> Config:
    cfg = Config()
    load().sph3_default_config(ctypes.byref(cfg))
    return cfg


def probe_fp32_rate(device: int = 0, stream=None) -> float:
    """Measured FP32 rate (TFLOP/s) of GPU `device`: packed FMA chains on every
    SM, timed with CUDA events (the walk kernels' roofline denominator)."""
    v = ctypes.c_double()
    check(load().sph3_probe_fp32_rate(int(device), ctypes.byref(v), stream), "probe_fp32_rate")
    return float(v.value)
