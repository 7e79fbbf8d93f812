"""Drop-in for the reference's Balsara-switch module sph_code/shear.py.

div/curl of v and the shear-corrected hydro acceleration and du/dt, on the
GPU through libsph3, with the settings of :mod:`sph_3_b200.libsx`.
"""
from __future__ import annotations

from . import libsx as _lx


def _divcurl(pos, v, rho, m, h, rows=None):
    ctx = _lx._context()
    ctx.set_particles(pos, m, vel=v, h=h)
    ctx.set_field("rho", rho)
    ctx.compute("divcurl")
    return (_lx._ret(None, pos, ctx, "divV", rows=rows), _lx._ret(None, pos, ctx, "curlV", rows=rows))


def div_curlVel(pos, v, rho, m, h):
    """(|div v|, |curl v|) per particle (shear.py:7-69)."""
    return _divcurl(pos, v, rho, m, h)


def div_curlVel_mpi(nbeg, nend, pos, v, rho, m, h):
    """Rows [nbeg, nend) of div_curlVel (shear.py:76-142)."""
    return _divcurl(pos, v, rho, m, h, rows=(nbeg, nend))


def getAcc_sph_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """Hydro acceleration with the Balsara factor (shear.py:149-235)."""
    return _lx._hydro(pos, v, rho, P, c, h, m, "acc_sph", "balsara", alpha, divV=divV, curlV=curlV)


def getAcc_sph_shear_mpi(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """Rows [nbeg, nend) of getAcc_sph_shear (shear.py:241-326)."""
    return _lx._hydro(pos, v, rho, P, c, h, m, "acc_sph", "balsara", alpha, divV=divV, curlV=curlV,
                      rows=(nbeg, nend))


def get_dU_shear(pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """du/dt with the Balsara factor (shear.py:332-406)."""
    return _lx._hydro(pos, v, rho, P, c, h, m, "dudt", "balsara", alpha, divV=divV, curlV=curlV)


def get_dU_shear_mpi(nbeg, nend, pos, v, rho, P, c, h, m, divV, curlV, alpha):
    """Rows [nbeg, nend) of get_dU_shear (shear.py:411-485)."""
    return _lx._hydro(pos, v, rho, P, c, h, m, "dudt", "balsara", alpha, divV=divV, curlV=curlV,
                      rows=(nbeg, nend))
