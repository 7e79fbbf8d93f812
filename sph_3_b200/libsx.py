"""Drop-in for the reference's CPU library sph_code/libsx.py.

Same function names, positional signatures, return shapes and dtypes; every
computation runs on the GPU through libsph3 (the octree walks replace the
reference's O(N^2) loops).  NumPy inputs give NumPy outputs; torch CUDA
tensors give torch CUDA tensors (no host copies).

Defaults reproduce the reference's results: FP64 arithmetic, the reference's
h rule (N_ngb = 50 +- 5, h -/+= 0.3 % per step), the signal-velocity
viscosity, and gravity (getAcc_g_smth*, getPE) as direct sums in the
reference's own summation order, which return its values bit for bit
(sph3_gravity_pairsum; O(N^2) work, as in the reference).  Options, set with
:func:`configure`:
  * ``grav_method="tree"`` switches gravity to the Barnes-Hut walk with
    ``theta`` (default 0.5; monopole + quadrupole), O(N log N);
  * the h search stops after ``h_max_iter`` steps of the 0.3 % rule (default
    10,000, a factor 1e13 in h) and flags SPH3_STATUS_H_NOT_CONVERGED, where
    the reference loops forever;
  * ``precision="mixed"`` switches to the FP32 cell-relative path.
Each call loads the particles, sorts them and builds the tree; for repeated
steps use :class:`sph_3_b200.Context` which keeps them resident.
"""
from __future__ import annotations

import numpy as np

from .context import Config, Context

_DEFAULT = Config(precision="fp64", h_mode="refstep", n_ngb=50, n_ngb_tol=5, h_max_iter=10000,
                  n_boot=50, theta=0.5, use_graph=False)
_cfg = _DEFAULT
_grav_method = "direct"  # "direct": reference-order sums; "tree": Barnes-Hut with theta
_ctx = None


def configure(grav_method=None, **kw):
    """Changes the settings used by every function of this module:
    ``grav_method`` ("direct" or "tree") and any :class:`Config` field."""
    global _cfg, _grav_method
    if grav_method is not None:
        if grav_method not in ("direct", "tree"):
            raise ValueError("grav_method must be 'direct' or 'tree'")
        _grav_method = grav_method
    _cfg = _cfg.replace(**kw)


def reset():
    global _cfg, _ctx, _grav_method
    _cfg = _DEFAULT
    _grav_method = "direct"
    if _ctx is not None:
        _ctx.close()
    _ctx = None


def _context(**over) -> Context:
    global _ctx
    cfg = _cfg.replace(**over)
    if _ctx is None:
        _ctx = Context(cfg)
    elif _ctx.config != cfg:
        _ctx.set_config(cfg)
    return _ctx


def _torch_like(x):
    return type(x).__module__.startswith("torch")


def _ret(arr_np, like, ctx=None, name=None, rows=None):
    """Field from the context as NumPy, or as a CUDA tensor when `like` is one."""
    if ctx is not None:
        if _torch_like(like) and getattr(like, "is_cuda", False):
            return ctx.get_field(name, rows=rows, device=True)
        return ctx.get_field(name, rows=rows)
    return arr_np


def _n(pos):
    return int(pos.shape[0])


def _ones(pos):
    if _torch_like(pos):
        import torch
        return torch.ones(_n(pos), dtype=torch.float64, device=pos.device)
    return np.ones(_n(pos))


# ------------------------------------------------------------ density, h
def getDensity(pos, m, h):
    """rho_i = sum_j m_j W(r_ij, (h_i + h_j) / 2) (libsx.py:10-44)."""
    ctx = _context()
    ctx.set_particles(pos, m, h=h)
    ctx.compute("density")
    return _ret(None, pos, ctx, "rho")


def getDensity_mpi(nbeg, nend, pos, m, h):
    """Rows [nbeg, nend) of getDensity (libsx.py:50-86)."""
    ctx = _context()
    ctx.set_particles(pos, m, h=h)
    ctx.compute("density", rows=(nbeg, nend))
    return _ret(None, pos, ctx, "rho", rows=(nbeg, nend))


def getPressure(rho, u, gama):
    """P = (gamma - 1) rho u (libsx.py:91-96), elementwise in the inputs' array type."""
    return (gama - 1.0) * rho * u


def h_smooth_fast(pos, h):
    """h with N(dist < 2h) in [N_ngb - 5, N_ngb + 5] (libsx.py:804-845)."""
    ctx = _context()
    ctx.set_particles(pos, _ones(pos), h=h)
    ctx.compute("h")
    return _ret(None, pos, ctx, "h")


def h_smooth_fast_mpi(nbeg, nend, pos, h):
    """Rows [nbeg, nend) of h_smooth_fast (libsx.py:852-902)."""
    ctx = _context()
    ctx.set_particles(pos, _ones(pos), h=h)
    ctx.compute("h", rows=(nbeg, nend))
    return _ret(None, pos, ctx, "h", rows=(nbeg, nend))


def smoothing_length_mpi(nbeg, nend, pos):
    """h = half the distance to the 51st nearest particle, self included
    (libsx.py:779-800)."""
    ctx = _context()
    ctx.set_particles(pos, _ones(pos))
    ctx.compute("boot_h", rows=(nbeg, nend))
    return _ret(None, pos, ctx, "h", rows=(nbeg, nend))


def do_smoothingX(poz):
    """h of each row of subpos: half the distance to its 51st-nearest row of
    pos, itself included when it is one of them (libsx.py:752-774)."""
    pos, subpos = poz
    same = subpos is pos
    if not same and not _torch_like(pos) and not _torch_like(subpos):
        same = np.shape(subpos) == np.shape(pos) and np.array_equal(np.asarray(subpos), np.asarray(pos))
    if not same and _torch_like(pos) and _torch_like(subpos):
        import torch
        same = subpos.shape == pos.shape and subpos.device == pos.device and bool(torch.equal(subpos, pos))
    if same:
        return smoothing_length_mpi(0, _n(pos), pos)
    ctx = _context()
    ctx.set_particles(pos, _ones(pos))
    out = ctx.kth_distance(subpos, 50, device=_torch_like(subpos) and getattr(subpos, "is_cuda", False))
    return out


# ------------------------------------------------------------ hydro
def _hydro(pos, v, rho, P, c, h, m, want, visc, alpha, beta=2.0, eta=0.1, divV=None, curlV=None,
           rows=None):
    ctx = _context(visc=visc, alpha=float(alpha), beta=float(beta), eta=float(eta))
    ctx.set_particles(pos, m, vel=v, h=h)
    ctx.set_field("rho", rho)
    ctx.set_field("P", P)
    ctx.set_field("c", c)
    if divV is not None:
        ctx.set_field("divV", divV)
        ctx.set_field("curlV", curlV)
    ctx.compute("acc_sph" if want == "acc_sph" else "dudt", rows=rows)
    return _ret(None, pos, ctx, want, rows=rows)


def getAcc_sph(pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """Hydro acceleration, signal-velocity viscosity (libsx.py:100-177)."""
    return _hydro(pos, v, rho, P, c, h, m, "acc_sph", "signal", alpha, beta, eta)


def getAcc_sph_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """Rows [nbeg, nend) of getAcc_sph (libsx.py:268-347)."""
    return _hydro(pos, v, rho, P, c, h, m, "acc_sph", "signal", alpha, beta, eta, rows=(nbeg, nend))


def getAcc_sph_mpiXXX(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """Monaghan & Gingold (1983) viscosity (libsx.py:183-262)."""
    return _hydro(pos, v, rho, P, c, h, m, "acc_sph", "mg83", alpha, beta, eta, rows=(nbeg, nend))


def get_dU(pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """du/dt, signal-velocity viscosity (libsx.py:353-421)."""
    return _hydro(pos, v, rho, P, c, h, m, "dudt", "signal", alpha, beta, eta)


def get_dU_mpi(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """Rows [nbeg, nend) of get_dU (libsx.py:496-564)."""
    return _hydro(pos, v, rho, P, c, h, m, "dudt", "signal", alpha, beta, eta, rows=(nbeg, nend))


def get_dU_mpiXXXX(nbeg, nend, pos, v, rho, P, c, h, m, gama, eta, alpha, beta):
    """Monaghan & Gingold (1983) du/dt (libsx.py:427-491)."""
    return _hydro(pos, v, rho, P, c, h, m, "dudt", "mg83", alpha, beta, eta, rows=(nbeg, nend))


# ------------------------------------------------------------ gravity, energy
def _eps_array(epsilon, pos):
    if np.ndim(epsilon) == 0 and not _torch_like(epsilon):
        return np.full(_n(pos), float(epsilon))
    return epsilon


def _gravity(pos, mass, G, epsilon, tree=True, rows=None):
    ctx = _context(G=float(G))
    ctx.set_particles(pos, mass, eps=_eps_array(epsilon, pos))
    if tree:
        ctx.compute("gravity", rows=rows)
    return ctx


def _grav_rows(pos, mass, G, epsilon, nbeg, nend, form="rows"):
    dev = _torch_like(pos) and getattr(pos, "is_cuda", False)
    if _grav_method == "direct":
        ctx = _gravity(pos, mass, G, epsilon, tree=False)
        return ctx.gravity_pairsum(form, nbeg, nend, device=dev)
    whole = nbeg == 0 and nend == _n(pos)
    ctx = _gravity(pos, mass, G, epsilon, rows=None if whole else (nbeg, nend))
    return _ret(None, pos, ctx, "acc_g", rows=(nbeg, nend))


def getAcc_g_smth(pos, mass, G, epsilon):
    """Spline-softened gravity (libsx.py:623-662)."""
    return _grav_rows(pos, mass, G, epsilon, 0, _n(pos))


def getAcc_g_smthx(pos, mass, G, epsilon):
    """Same field as getAcc_g_smth (libsx.py:710-747)."""
    return getAcc_g_smth(pos, mass, G, epsilon)


def getAcc_g_smth_mpi(nbeg, nend, pos, mass, G, epsilon):
    """Rows [nbeg, nend) of the field (libsx.py:667-705)."""
    return _grav_rows(pos, mass, G, epsilon, nbeg, nend)


def getAcc_g_smth_mimj_mpi(nbeg, nend, pos, mass, G, epsilon):
    """The (N, 3) partial field of libsx.py:908-947: the j > i terms of rows
    i in [nbeg, nend) and their reactions on the rows j > i, so the sum over a
    row partition is the full field.  With grav_method="tree" it is instead
    the full acceleration on rows [nbeg, nend) and zero elsewhere (the same
    sum over a partition)."""
    if _grav_method == "direct":
        return _grav_rows(pos, mass, G, epsilon, nbeg, nend, form="mimj")
    part = _grav_rows(pos, mass, G, epsilon, nbeg, nend)
    if _torch_like(part):
        import torch
        out = torch.zeros((_n(pos), 3), dtype=torch.float64, device=part.device)
    else:
        out = np.zeros((_n(pos), 3))
    out[nbeg:nend] = part
    return out


def getKE(v, m):
    """sum 0.5 m v^2 (libsx.py:569-579), FP64 sum on the GPU."""
    ctx = _context()
    zeros = np.zeros((_n(v), 3)) if not _torch_like(v) else v * 0.0
    ctx.set_particles(zeros, m, vel=v)
    return float(ctx.energy()["KE"])


def getPE(pos, m, G, epsilon):
    """Softened potential energy (libsx.py:583-620): FP64 pair sums in the
    reference's row order (grav_method="direct"), or 1/2 sum m_i phi_i of the
    Barnes-Hut walk ("tree")."""
    if _grav_method == "direct":
        return _gravity(pos, m, G, epsilon, tree=False).potential_pairsum()
    ctx = _gravity(pos, m, G, epsilon)
    return float(ctx.energy()["PE"])
