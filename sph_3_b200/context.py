"""Host-side API around one sph3 context: NumPy arrays (host) or torch CUDA
tensors (zero-copy, stream-ordered) in, the same kinds out.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, fields
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import C, check

FIELDS = {
    "pos": (C["SPH3_FIELD_POS"], 3), "vel": (C["SPH3_FIELD_VEL"], 3), "m": (C["SPH3_FIELD_MASS"], 1),
    "u": (C["SPH3_FIELD_U"], 1), "h": (C["SPH3_FIELD_H"], 1), "eps": (C["SPH3_FIELD_EPS"], 1),
    "rho": (C["SPH3_FIELD_RHO"], 1), "P": (C["SPH3_FIELD_P"], 1), "c": (C["SPH3_FIELD_C"], 1),
    "divV": (C["SPH3_FIELD_DIVV"], 1), "curlV": (C["SPH3_FIELD_CURLV"], 1),
    "acc": (C["SPH3_FIELD_ACC"], 3), "acc_g": (C["SPH3_FIELD_ACC_G"], 3),
    "acc_sph": (C["SPH3_FIELD_ACC_SPH"], 3), "dudt": (C["SPH3_FIELD_DUDT"], 1),
    "dudt_prev": (C["SPH3_FIELD_DUDT_PREV"], 1), "phi": (C["SPH3_FIELD_PHI"], 1),
    "nngb": (C["SPH3_FIELD_NNGB"], 1), "balsara": (C["SPH3_FIELD_BALSARA"], 1),
    "u_prev": (C["SPH3_FIELD_U_PREV"], 1), "vsig": (C["SPH3_FIELD_VSIG"], 1),
    "dt": (C["SPH3_FIELD_DT"], 1), "dhdt": (C["SPH3_FIELD_DHDT"], 1),
}

DO = {k[len("SPH3_DO_"):].lower(): v for k, v in C.items() if k.startswith("SPH3_DO_")}
STATUS_BITS = {k[len("SPH3_STATUS_"):]: v for k, v in C.items() if k.startswith("SPH3_STATUS_")}

_PREC = {"mixed": C["SPH3_PREC_MIXED"], "fp64": C["SPH3_PREC_FP64"]}
_HMODE = {"newton": C["SPH3_H_NEWTON"], "refstep": C["SPH3_H_REFSTEP"]}
_VISC = {"signal": C["SPH3_VISC_SIGNAL"], "mg83": C["SPH3_VISC_MG83"], "balsara": C["SPH3_VISC_BALSARA"]}
_ORDER = {"serial": C["SPH3_ORDER_SERIAL"], "mpi4": C["SPH3_ORDER_MPI4"]}
_MAC = {"bh": C["SPH3_MAC_BH"], "bh_offset": C["SPH3_MAC_BH_OFFSET"]}


@dataclass
class Config:
    """Physics and numerics of a context (defaults: the Evrard benchmark setup)."""
    precision: str = "mixed"       # "mixed" | "fp64"
    h_mode: str = "newton"         # "newton" | "refstep" (the reference's +-0.3 % rule)
    visc: str = "signal"           # "signal" | "mg83" | "balsara"
    step_order: str = "serial"     # "serial" (sph_serial.py) | "mpi4" (sph_mpi4_v4.py)
    n_ngb: int = 64
    n_ngb_tol: int = 5
    h_max_iter: int = 64
    n_boot: int = 50
    leaf_size: int = 16
    stack_cap: int = 768
    max_level: int = 16
    gravity: bool = True
    quadrupole: bool = True
    use_graph: bool = True
    timing: bool = False
    walk_warps: int = 4            # warps per walk block (1, 2, 4, 8)
    list_cap: int = 128            # neighbour-list slots per particle for the hydro pass (0: walk)
    mac: str = "bh"                # multipole acceptance: "bh" (d > s/theta) | "bh_offset" (+ com offset)
    eps_from_h: bool = False       # softening eps = h after every h search (reference GPU driver option)
    step_potential: bool = False   # every step's gravity also computes the potential (else on demand)
    gamma: float = 5.0 / 3.0
    alpha: float = 1.0
    beta: float = 2.0
    eta: float = 0.1
    G: float = 1.0
    theta: float = 0.5
    eps: float = 0.01
    box: Sequence[float] = (0.0, 0.0, 0.0)

    def to_c(self) -> _lib.Config:
        c = _lib.default_config()
        c.precision = _PREC[self.precision]
        c.h_mode = _HMODE[self.h_mode]
        c.visc = _VISC[self.visc]
        c.step_order = _ORDER[self.step_order]
        c.mac = _MAC[self.mac]
        for name in ("n_ngb", "n_ngb_tol", "h_max_iter", "n_boot", "leaf_size", "stack_cap", "max_level",
                     "walk_warps", "list_cap"):
            setattr(c, name, int(getattr(self, name)))
        for name in ("gravity", "quadrupole", "use_graph", "timing", "eps_from_h", "step_potential"):
            setattr(c, name, 1 if getattr(self, name) else 0)
        for name in ("gamma", "alpha", "beta", "eta", "G", "theta", "eps"):
            setattr(c, name, float(getattr(self, name)))
        for k in range(3):
            c.box[k] = float(self.box[k])
        return c

    def replace(self, **kw) -> "Config":
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d.update(kw)
        return Config(**d)


def _is_torch(a):
    return type(a).__module__.startswith("torch")


# CUDA's handle of the legacy default stream (cudaStreamLegacy)
_CUDA_STREAM_LEGACY = 1


def _stream_ptr():
    """torch's current stream as a cudaStream_t for the C ABI.  torch reports
    its legacy default stream as handle 0, which the C ABI reads as "the
    context's own stream" (not ordered with torch's work), so that one is
    passed as cudaStreamLegacy."""
    import torch
    h = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(h if h else _CUDA_STREAM_LEGACY)


class Context:
    """One device-resident particle set (or batch of systems) and its tree.

    Arrays may be NumPy (host; copied in and out synchronously) or torch CUDA
    float64 tensors (used in place, ordered on torch's current stream).
    Particle order is always the caller's."""

    def __init__(self, config: Optional[Config] = None, device: int = -1):
        self.lib = _lib.load()
        self.config = config or Config()
        self._ptr = ctypes.c_void_p()
        cfg = self.config.to_c()
        check(self.lib.sph3_ctx_create(ctypes.byref(cfg), int(device), ctypes.byref(self._ptr)),
              "ctx_create")
        self.n = 0
        self.ncloud = 1
        self._keep = []

    # ------------------------------------------------------------ lifetime
    def close(self):
        if self._ptr:
            self.lib.sph3_ctx_destroy(self._ptr)
            self._ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_config(self, config: Config):
        cfg = config.to_c()
        check(self.lib.sph3_set_config(self._ptr, ctypes.byref(cfg)), "set_config")
        self.config = config

    # ------------------------------------------------------------ arrays
    def _arg(self, a, ncomp, n=None):
        """-> (pointer, on_device, keepalive)."""
        if a is None:
            return None, 0, None
        if _is_torch(a):
            import torch
            if a.is_cuda:
                t = a.detach().to(torch.float64).contiguous()
                if n is not None and t.numel() != n * ncomp:
                    raise ValueError("expected %d values, got %d" % (n * ncomp, t.numel()))
                return ctypes.c_void_p(t.data_ptr()), 1, t
            a = a.detach().cpu().numpy()
        arr = np.ascontiguousarray(a, dtype=np.float64)
        if n is not None and arr.size != n * ncomp:
            if arr.size == 1 and ncomp == 1:
                arr = np.full(n, float(arr.reshape(-1)[0]))
            else:
                raise ValueError("expected %d values, got %d" % (n * ncomp, arr.size))
        return arr.ctypes.data_as(ctypes.c_void_p), 0, arr

    def _stream(self, on_device):
        return _stream_ptr() if on_device else None

    def set_clouds(self, counts):
        arr = np.ascontiguousarray(counts, dtype=np.int64)
        check(self.lib.sph3_set_clouds(self._ptr, arr.ctypes.data_as(ctypes.c_void_p), int(arr.size)),
              "set_clouds")
        self.ncloud = int(arr.size)

    def set_particles(self, pos, m, vel=None, u=None, h=None, eps=None):
        n = int(pos.shape[0]) if hasattr(pos, "shape") else len(pos)
        # C order: pos, vel, mass, u, h, eps
        args = [self._arg(pos, 3, n), self._arg(vel, 3, n), self._arg(m, 1, n), self._arg(u, 1, n),
                self._arg(h, 1, n), self._arg(eps, 1, n)]
        devs = {a[1] for a in args if a[0] is not None}
        if len(devs) > 1:
            raise ValueError("mix of host arrays and CUDA tensors")
        on_dev = devs.pop() if devs else 0
        ptrs = [a[0] for a in args]
        check(self.lib.sph3_set_particles(self._ptr, n, *ptrs, on_dev, self._stream(on_dev)),
              "set_particles")
        self.n = n
        return self

    def set_field(self, name, arr):
        fid, nc = FIELDS[name]
        p, on_dev, keep = self._arg(arr, nc, self.n)
        check(self.lib.sph3_set_field(self._ptr, fid, p, on_dev, self._stream(on_dev)), "set_field " + name)
        del keep

    def get_field(self, name, rows=None, device=False, out=None):
        """Field values (caller's order).  rows: (begin, end) slice or None.
        device=True returns a torch CUDA tensor.  out: a C-contiguous float64
        host array (NumPy, or a torch CPU tensor, e.g. page-locked) of the
        field's shape to copy into instead of a new array."""
        fid, nc = FIELDS[name]
        b, e = (0, self.n) if rows is None else (int(rows[0]), int(rows[1]))
        shape = (e - b, nc) if nc > 1 else (e - b,)
        if out is not None:
            if hasattr(out, "data_ptr"):  # torch CPU tensor
                ok = (not out.is_cuda and out.is_contiguous() and str(out.dtype) == "torch.float64"
                      and tuple(out.shape) == shape)
                ptr = out.data_ptr()
            else:
                ok = (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                      and out.shape == shape)
                ptr = out.ctypes.data if ok else 0
            if not ok:
                raise ValueError("get_field out= must be a C-contiguous float64 host array of shape %s" % (shape,))
            check(self.lib.sph3_get_field(self._ptr, fid, ctypes.c_void_p(ptr), b, e, 0, None),
                  "get_field " + name)
            return out
        if device:
            import torch
            out = torch.empty(shape, dtype=torch.float64, device="cuda")
            check(self.lib.sph3_get_field(self._ptr, fid, ctypes.c_void_p(out.data_ptr()), b, e, 1,
                                          _stream_ptr()), "get_field " + name)
            return out
        out = np.empty(shape, dtype=np.float64)
        check(self.lib.sph3_get_field(self._ptr, fid, out.ctypes.data_as(ctypes.c_void_p), b, e, 0, None),
              "get_field " + name)
        return out

    # ------------------------------------------------------------ passes
    def compute(self, *what, rows=None):
        """Run the named passes; rows=(begin, end) runs the walks only for
        those rows in the caller's order (sph3_compute_rows: the other rows'
        pair results are left undefined)."""
        mask = 0
        for w in what:
            mask |= DO[w] if isinstance(w, str) else int(w)
        if rows is None:
            check(self.lib.sph3_compute(self._ptr, mask, None), "compute")
        else:
            b, e = int(rows[0]), int(rows[1])
            check(self.lib.sph3_compute_rows(self._ptr, mask, b, e, None), "compute_rows")

    def first_step(self, dt):
        check(self.lib.sph3_first_step(self._ptr, float(dt), None), "first_step")

    def step(self, dt, nsteps=1, stream=None):
        st = ctypes.c_void_p(stream) if stream is not None else None
        check(self.lib.sph3_step(self._ptr, float(dt), int(nsteps), st), "step")

    def step_io(self, dt, inputs, outputs, nsteps=1):
        """nsteps steps with the state moved in from and out to host arrays in
        one call (sph3_step_io): inputs {field: array}, outputs {field:
        C-contiguous float64 host array to fill, e.g. page-locked torch CPU
        tensors}; transfers overlap the step."""
        def host_ptr(a, name, shape):
            if hasattr(a, "data_ptr"):
                ok = (not a.is_cuda and a.is_contiguous() and str(a.dtype) == "torch.float64"
                      and tuple(a.shape) in (shape, (self.n * FIELDS[name][1],)))
                return a.data_ptr() if ok else None
            a_ok = (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                    and a.size == self.n * FIELDS[name][1])
            return a.ctypes.data if a_ok else None

        def shape_of(name):
            nc = FIELDS[name][1]
            return (self.n, nc) if nc > 1 else (self.n,)

        keep = []
        in_f, in_p = [], []
        for name, a in inputs.items():
            if not hasattr(a, "data_ptr"):
                a = np.ascontiguousarray(a, dtype=np.float64)
                keep.append(a)
            p = host_ptr(a, name, shape_of(name))
            if p is None:
                raise ValueError("step_io input %s must be a float64 host array of shape %s" % (name, shape_of(name)))
            in_f.append(FIELDS[name][0])
            in_p.append(p)
        out_f, out_p = [], []
        for name, a in outputs.items():
            p = host_ptr(a, name, shape_of(name))
            if p is None:
                raise ValueError("step_io output %s must be a C-contiguous float64 host array of shape %s"
                                 % (name, shape_of(name)))
            out_f.append(FIELDS[name][0])
            out_p.append(p)
        fi = (ctypes.c_int32 * max(1, len(in_f)))(*in_f)
        pi = (ctypes.c_void_p * max(1, len(in_p)))(*in_p)
        fo = (ctypes.c_int32 * max(1, len(out_f)))(*out_f)
        po = (ctypes.c_void_p * max(1, len(out_p)))(*out_p)
        check(self.lib.sph3_step_io(self._ptr, float(dt), int(nsteps), len(in_f), fi, pi, len(out_f), fo, po, None),
              "step_io")
        del keep

    def energy(self):
        out = np.zeros(8)
        check(self.lib.sph3_energy(self._ptr, out.ctypes.data_as(ctypes.c_void_p), None), "energy")
        return dict(KE=out[0], U=out[1], PE=out[2], E=out[3], px=out[4], py=out[5], pz=out[6], M=out[7])

    def status(self, clear=False):
        v = ctypes.c_uint32()
        check(self.lib.sph3_status(self._ptr, ctypes.byref(v), 1 if clear else 0), "status")
        return int(v.value)

    def status_names(self, clear=False):
        s = self.status(clear)
        return [k for k, b in STATUS_BITS.items() if s & b]

    def counters(self, clear=False):
        out = np.zeros(16, dtype=np.int64)
        check(self.lib.sph3_counters(self._ptr, out.ctypes.data_as(ctypes.c_void_p), 1 if clear else 0),
              "counters")
        keys = ["grav_node", "grav_part", "density_pairs", "hydro_pairs", "h_pairs", "h_passes",
                "tree_nodes", "tree_leaves", "visits_h", "visits_density", "visits_hydro", "visits_gravity",
                "walk_max_iter", "walk_max_where", "grav_groups"]
        return dict(zip(keys, out.tolist()))

    def timestep(self, c_cfl=0.25, all_pairs=False):
        """Per-particle time steps of the reference's criterion (see sph3_timestep in
        include/sph3.h); returns (dt per particle in the caller's order, min dt)."""
        v = ctypes.c_double()
        check(self.lib.sph3_timestep(self._ptr, float(c_cfl), 1 if all_pairs else 0, ctypes.byref(v), None),
              "timestep")
        return self.get_field("dt"), float(v.value)

    def set_cooling(self, table=None, units=None):
        """Every later step applies the cooling table to u right after the u
        update (hcoolingZ after u_updater in the production driver); None
        turns it off.  `table` is a :class:`sph_3_b200.cooling.CoolTable` on
        this context's GPU, `units` a :class:`sph_3_b200.cooling.Units`."""
        if table is None:
            check(self.lib.sph3_set_cooling(self._ptr, None, None), "set_cooling")
            self._cool = None
            return
        cu = units.to_c()
        check(self.lib.sph3_set_cooling(self._ptr, table.handle, ctypes.byref(cu)), "set_cooling")
        self._cool = table  # the context uses the table until cooling is turned off

    def cool_now(self, dt):
        """Applies the cooling table set by :meth:`set_cooling` once to the current state."""
        check(self.lib.sph3_cool_now(self._ptr, float(dt), None), "cool_now")

    def ionfrac(self):
        """Species fractions of the last cooled step, (n, N_M) float32, caller's order."""
        tab = getattr(self, "_cool", None)
        if tab is None:
            raise RuntimeError("no cooling table is set")
        out = np.empty((self.n, tab.n_species), np.float32)
        check(self.lib.sph3_get_ionfrac(self._ptr, out.ctypes.data_as(ctypes.c_void_p), tab.n_species),
              "get_ionfrac")
        return out

    def kernels_per_step(self):
        """Kernel launches per step of the captured step graph (-1 before capture)."""
        v = ctypes.c_int64()
        check(self.lib.sph3_kernels_per_step(self._ptr, ctypes.byref(v)), "kernels_per_step")
        return int(v.value)

    def phase_times(self, clear=False):
        out = np.zeros(9)
        check(self.lib.sph3_phase_times(self._ptr, out.ctypes.data_as(ctypes.c_void_p), 1 if clear else 0),
              "phase_times")
        keys = ["kick_drift_keys", "sort", "gather", "tree", "h", "density", "gravity", "hydro", "kick_u"]
        return dict(zip(keys, out.tolist()))

    # ------------------------------------------------------------ checks
    def gravity_direct_rows(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        acc = np.zeros((rows.size, 3))
        phi = np.zeros(rows.size)
        check(self.lib.sph3_gravity_direct_rows(self._ptr, rows.ctypes.data_as(ctypes.c_void_p), rows.size,
                                                acc.ctypes.data_as(ctypes.c_void_p),
                                                phi.ctypes.data_as(ctypes.c_void_p)), "gravity_direct_rows")
        return acc, phi

    def gravity_pairsum(self, form="rows", nbeg=0, nend=None, device=False):
        """Reference-order FP64 gravity (sph3_gravity_pairsum): form "rows" gives
        rows [nbeg, nend) of getAcc_g_smth / _mpi / x, form "mimj" the (n, 3)
        partial array of getAcc_g_smth_mimj_mpi(nbeg, nend, ...)."""
        nend = self.n if nend is None else int(nend)
        nbeg = int(nbeg)
        code = {"rows": C["SPH3_GSUM_ROWS"], "mimj": C["SPH3_GSUM_MIMJ"]}[form]
        rows = (nend - nbeg) if form == "rows" else self.n
        if device:
            import torch
            out = torch.empty((max(rows, 0), 3), dtype=torch.float64, device="cuda")
            check(self.lib.sph3_gravity_pairsum(self._ptr, code, nbeg, nend, ctypes.c_void_p(out.data_ptr()), 1,
                                                _stream_ptr()), "gravity_pairsum")
            return out
        out = np.zeros((max(rows, 0), 3))
        check(self.lib.sph3_gravity_pairsum(self._ptr, code, nbeg, nend, out.ctypes.data_as(ctypes.c_void_p), 0,
                                            None), "gravity_pairsum")
        return out

    def potential_pairsum(self):
        """getPE as FP64 pair sums in the reference's row order (sph3_potential_pairsum)."""
        v = ctypes.c_double()
        check(self.lib.sph3_potential_pairsum(self._ptr, ctypes.byref(v), None), "potential_pairsum")
        return float(v.value)

    def kth_distance(self, qpos, k=50, device=False):
        """0.5 x the k-th (0-based) sorted distance from each query point to the
        loaded particles (sph3_kth_distance; do_smoothingX with k = 50)."""
        if _is_torch(qpos) and qpos.is_cuda:
            import torch
            q = qpos.detach().to(torch.float64).contiguous()
            m = int(q.shape[0])
            out = torch.empty(m, dtype=torch.float64, device=q.device)
            check(self.lib.sph3_kth_distance(self._ptr, ctypes.c_void_p(q.data_ptr()), m, int(k),
                                             ctypes.c_void_p(out.data_ptr()), 1, _stream_ptr()), "kth_distance")
            return out
        if _is_torch(qpos):
            qpos = qpos.detach().cpu().numpy()
        q = np.ascontiguousarray(qpos, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(q.shape[0])
        check(self.lib.sph3_kth_distance(self._ptr, q.ctypes.data_as(ctypes.c_void_p), q.shape[0], int(k),
                                         out.ctypes.data_as(ctypes.c_void_p), 0, None), "kth_distance")
        return out

    def neighbours(self, rows, cap=None):
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cap = int(cap if cap is not None else max(1, rows.size) * 512)
        off = np.zeros(rows.size + 1, dtype=np.int64)
        idx = np.zeros(max(cap, 1), dtype=np.int64)
        check(self.lib.sph3_neighbours(self._ptr, rows.ctypes.data_as(ctypes.c_void_p), rows.size,
                                       off.ctypes.data_as(ctypes.c_void_p), idx.ctypes.data_as(ctypes.c_void_p),
                                       cap), "neighbours")
        return [idx[off[k]:off[k + 1]].copy() for k in range(rows.size)]

    def pair_lists(self, rows, cap=None):
        """The mixed path's kept pairs (sph3_pair_lists) of the listed rows, caller indices, ascending."""
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cap = int(cap if cap is not None else max(1, rows.size) * 1024)
        off = np.zeros(rows.size + 1, dtype=np.int64)
        idx = np.zeros(max(cap, 1), dtype=np.int64)
        check(self.lib.sph3_pair_lists(self._ptr, rows.ctypes.data_as(ctypes.c_void_p), rows.size,
                                       off.ctypes.data_as(ctypes.c_void_p), idx.ctypes.data_as(ctypes.c_void_p),
                                       cap), "pair_lists")
        return [idx[off[k]:off[k + 1]].copy() for k in range(rows.size)]

    def morton_order(self):
        order = np.zeros(self.n, dtype=np.int64)
        keys = np.zeros(self.n, dtype=np.uint64)
        check(self.lib.sph3_morton_order(self._ptr, order.ctypes.data_as(ctypes.c_void_p),
                                         keys.ctypes.data_as(ctypes.c_void_p)), "morton_order")
        return order, keys
