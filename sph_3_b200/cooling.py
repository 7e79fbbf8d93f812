"""Table-driven heating/cooling of the gas: the production driver's step after
the u update (hcoolingZ, Particles_in_BH_Tree_III/Evrard_Collapse_2024/
hfvCLibs_v7_hfv_v8.1.h:1433-1623, launched after u_updater at
Main_Code/hfvGpuSphBHtree_newCool_v8.cu:1552).

The table is the reference's coolHeatGridJan2024.bin (read at
Main_Code/hfvGpuSphBHtree_newCool_v8.cu:40-80): six int32 dimensions
N_kpc, N_T, N_nH, N_Z, N_M, N_t, then float32 arrays kpc, nH, Z, T, t, uEvol
[kpc][T][nH][Z][t], muArr (same shape), metalz [kpc][T][nH][Z][M][t] and
uArr [kpc][T][nH][Z].  The table itself (CHIMES output) is not part of the
reference repository; :func:`read_table` loads one where a user has it and
:func:`seeded_table` makes a table of the same layout for tests and
benchmarks.

Three ways to run it, all through ``libsph3.so``:

* :func:`hcooling` on the reference's float arrays (torch CUDA tensors in
  place, or NumPy arrays copied through the GPU);
* :meth:`sph_3_b200.Context.set_cooling`: every step applies the table right
  after the u update, inside the captured step;
* :meth:`sph_3_b200.Context.cool_now`: once, on the current state.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check

_DIM_NAMES = ("N_kpc", "N_T", "N_nH", "N_Z", "N_M", "N_t")


@dataclass
class Units:
    """The unit conversions of the reference's params.txt (float there, float
    here) and the table's metallicity row (the reference fixes 1: [Z/H] = -1)."""
    unit_density_cgs: float
    unit_time_s: float
    unit_u_cgs: float
    unit_length_cm: float
    kpc_cm: float = 3.086e21
    z_index: int = 1

    def to_c(self) -> "_lib.CoolUnits":
        return _lib.CoolUnits(self.unit_density_cgs, self.unit_time_s, self.unit_u_cgs, self.unit_length_cm,
                              self.kpc_cm, int(self.z_index))

    def as_tuple(self):
        return (self.unit_density_cgs, self.unit_time_s, self.unit_u_cgs, self.unit_length_cm, self.kpc_cm)


def _shapes(dims):
    nk, nT, nh, nZ, nM, nt = (int(d) for d in dims)
    return {"kpc": (nk,), "nH": (nh,), "Z": (nZ,), "T": (nT,), "t": (nt,),
            "uEvol": (nk, nT, nh, nZ, nt), "muArr": (nk, nT, nh, nZ, nt),
            "metalz": (nk, nT, nh, nZ, nM, nt), "uArr": (nk, nT, nh, nZ)}


_ORDER = ("kpc", "nH", "Z", "T", "t", "uEvol", "muArr", "metalz", "uArr")


def read_table(path) -> dict:
    """Reads a cooling table file in the reference's layout; returns a dict
    with ``dims`` (int32[6]) and the float32 arrays by the reference's names."""
    with open(path, "rb") as fh:
        raw = fh.read()
    dims = np.frombuffer(raw, dtype=np.int32, count=6).copy()
    if np.any(dims <= 0):
        raise ValueError("bad cooling-table header %s" % dims)
    out = {"dims": dims}
    at = 24
    for name in _ORDER:
        shape = _shapes(dims)[name]
        cnt = int(np.prod(shape))
        if at + 4 * cnt > len(raw):
            raise ValueError("cooling table %s is short (%s)" % (path, name))
        out[name] = np.frombuffer(raw, dtype=np.float32, count=cnt, offset=at).reshape(shape).copy()
        at += 4 * cnt
    return out


def write_table(path, table: dict) -> None:
    """Writes a table dict (as :func:`read_table` returns) in the reference's layout."""
    dims = np.asarray(table["dims"], dtype=np.int32)
    with open(path, "wb") as fh:
        fh.write(dims.tobytes())
        for name in _ORDER:
            a = np.asarray(table.get(name, np.zeros(_shapes(dims)[name], np.float32)), dtype=np.float32)
            if a.shape != _shapes(dims)[name]:
                raise ValueError("%s has shape %s, expected %s" % (name, a.shape, _shapes(dims)[name]))
            fh.write(np.ascontiguousarray(a).tobytes())


def seeded_table(seed=0, dims=(24, 60, 40, 3, 12, 30)) -> dict:
    """A table of the reference's layout with physically ordered values, for
    tests and benchmarks (the CHIMES tables are not distributed with the
    reference): ascending kpc, nH (cm^-3) and elapsed-time (s) grids; u(T)
    rising with T in every column; u after time t relaxing towards an
    equilibrium that depends on kpc and nH; species fractions in [0, 1]."""
    rng = np.random.default_rng(seed)
    nk, nT, nh, nZ, nM, nt = dims
    kpc = np.sort(rng.uniform(0.0, 2.0, nk)).astype(np.float32)
    kpc[0] = 0.0
    nH = np.logspace(-4, 4, nh).astype(np.float32)
    Z = np.array([-2.0, -1.0, 0.0][:nZ] + [0.0] * max(0, nZ - 3), np.float32)
    T = np.logspace(1, 8, nT).astype(np.float32)
    t = np.concatenate([[0.0], np.logspace(7, 14, nt - 1)]).astype(np.float32)
    mu = 0.6 + 0.6 * rng.random((nk, nT, nh, nZ))
    uarr = (1.5 * 1.380649e-16 * T[None, :, None, None] / (mu * 1.6726e-24)).astype(np.float32)
    # keep every T column strictly increasing after the random mu
    uarr = np.maximum.accumulate(uarr, axis=1) * (1.0 + 1e-3 * np.arange(nT, dtype=np.float32))[None, :, None, None]
    ueq = uarr[:, nT // 3: nT // 3 + 1] * (1.0 + 0.5 * rng.random((nk, 1, nh, nZ)))
    tau = 1e10 / (1.0 + nH[None, None, :, None]) * (1.0 + rng.random((nk, nT, nh, nZ)))
    frac = np.exp(-t[None, None, None, None, :] / tau[..., None])
    uevol = (ueq[..., None] + (uarr[..., None] - ueq[..., None]) * frac).astype(np.float32)
    metalz = rng.random((nk, nT, nh, nZ, nM, nt)).astype(np.float32)
    muarr = np.broadcast_to(mu[..., None], uevol.shape).astype(np.float32)
    return {"dims": np.array(dims, np.int32), "kpc": kpc, "nH": nH, "Z": Z, "T": T, "t": t,
            "uEvol": uevol, "muArr": muarr,
            "metalz": metalz, "uArr": uarr}


class CoolTable:
    """A cooling table resident on one GPU (sph3_cool_table)."""

    def __init__(self, table: dict, device: int = -1):
        import torch
        if device < 0:
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        self.device = int(device)
        self.dims = np.ascontiguousarray(table["dims"], dtype=np.int32)
        self.n_species = int(self.dims[4])
        arrs = [np.ascontiguousarray(table[k], dtype=np.float32) for k in ("kpc", "nH", "t", "uEvol", "metalz", "uArr")]
        h = ctypes.c_void_p()
        lib = _lib.load()
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        check(lib.sph3_cool_table_create(self.device, vp(self.dims), *[vp(a) for a in arrs], ctypes.byref(h)),
              "cool_table_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def monotone(self):
        """(kpc, nH, t grids, u columns) non-decreasing, as the library found them."""
        d = (ctypes.c_int32 * 6)()
        m = (ctypes.c_int32 * 4)()
        check(_lib.load().sph3_cool_table_dims(self._h, d, m), "cool_table_dims")
        return tuple(bool(x) for x in m)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().sph3_cool_table_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hcooling(table: CoolTable, units: Units, dt, u, rho, pos, typ=None, ionfrac=True, stream=None):
    """hcoolingZ on the reference's float arrays.  torch float32 CUDA tensors:
    u is updated in place and the ion fractions are returned as a CUDA tensor
    (stream-ordered, no synchronisation).  NumPy arrays: copied through the
    GPU; returns (u_new, ionfrac) as NumPy arrays.  pos: (n, 3), or the
    reference's separate x, y, z arrays as a tuple; typ: int32 (0 = gas) or
    None (all gas)."""
    import torch
    lib = _lib.load()
    on_dev = isinstance(u, torch.Tensor) and u.is_cuda
    dev = torch.device("cuda", table.device)
    split = isinstance(pos, (tuple, list))
    if on_dev:
        ut, rt, tt = u, rho, typ
        xs = list(pos) if split else [pos[:, k].contiguous() for k in range(3)]
    else:
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)  # noqa: E731
        ut, rt = f32(u), f32(rho)
        p = np.stack([np.asarray(a) for a in pos], axis=1) if split else np.asarray(pos)
        xs = [f32(p[:, k]) for k in range(3)]
        tt = None if typ is None else torch.as_tensor(np.ascontiguousarray(typ, dtype=np.int32)).to(dev)
    n = ut.shape[0]
    for name, a in (("u", ut), ("rho", rt), ("x", xs[0]), ("y", xs[1]), ("z", xs[2])):
        if a.dtype != torch.float32 or not a.is_cuda or not a.is_contiguous() or a.shape != (n,):
            raise TypeError("%s must be a contiguous float32 tensor of n entries on the GPU" % name)
    if tt is not None and (tt.dtype != torch.int32 or tt.shape != (n,) or not tt.is_contiguous()):
        raise TypeError("typ must be a contiguous int32 tensor of n entries")
    ion = torch.empty((n, table.n_species), dtype=torch.float32, device=ut.device) if ionfrac else None
    st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(ut.device).cuda_stream)
    cu = units.to_c()
    P = lambda t: ctypes.c_void_p(0 if t is None else t.data_ptr())  # noqa: E731
    with torch.cuda.device(ut.device):
        check(lib.sph3_hcooling(table.handle, ctypes.byref(cu), ctypes.c_float(dt), n, P(tt), P(ut), P(rt),
                                P(xs[0]), P(xs[1]), P(xs[2]), P(ion), None, st), "hcooling")
    if on_dev:
        return ut, ion
    torch.cuda.synchronize(ut.device)
    return ut.cpu().numpy(), (ion.cpu().numpy() if ion is not None else None)
