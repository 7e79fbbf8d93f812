"""sph3_compute_rows: the walks run only for a slice of rows in the caller's
order (the *_mpi forms of sph_code/libsx.py, one slice per rank of
sph_mpi4_v4.py), and the slice's results equal the full computation's bit
for bit (a walk group's results depend only on the group)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 20000


def _state(seed=5):
    from sph_3_b200.ic import evrard
    ic = evrard(N, seed=seed)
    rng = np.random.default_rng(seed)
    ic["vel"] = rng.normal(scale=0.05, size=(N, 3))
    return ic


def _ctx(ic, **cfg):
    from sph_3_b200 import Config, Context
    ctx = Context(Config(**cfg))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h")
    ctx.compute("h", "density")
    return ctx


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("rows", [(0, 1), (4321, 9876), (N - 700, N)])
def test_rows_equal_full(prec, rows):
    ic = _state()
    full = _ctx(ic, precision=prec)
    part = _ctx(ic, precision=prec)
    b, e = rows
    state = {f: full.get_field(f) for f in ("h", "rho", "P", "c")}
    # h search and density
    for what, field in (("h", "h"), ("density", "rho"), ("boot_h", "h")):
        for ctx in (full, part):
            ctx.set_field("h", state["h"])
        full.compute(what)
        part.compute(what, rows=rows)
        assert np.array_equal(part.get_field(field, rows=rows), full.get_field(field, rows=rows)), what
    # hydro (acceleration and du/dt) from the same rho, P, c
    for ctx in (full, part):
        for f in ("h", "rho", "P", "c"):
            ctx.set_field(f, state[f])
    full.compute("acc_sph", "dudt")
    part.compute("acc_sph", "dudt", rows=rows)
    for f in ("acc_sph", "dudt"):
        assert np.array_equal(part.get_field(f, rows=rows), full.get_field(f, rows=rows)), f
    # Barnes-Hut gravity
    full.compute("gravity")
    part.compute("gravity", rows=rows)
    assert np.array_equal(part.get_field("acc_g", rows=rows), full.get_field("acc_g", rows=rows))
    assert full.status() == 0 and part.status() == 0
    # a full step after a row-restricted call runs on complete data
    for ctx in (full, part):
        ctx.set_field("h", state["h"])
    full.first_step(1e-3)
    part.first_step(1e-3)
    assert np.array_equal(part.get_field("pos"), full.get_field("pos"))
    assert np.array_equal(part.get_field("rho"), full.get_field("rho"))
    full.close()
    part.close()


def test_rows_bad_arguments():
    from sph_3_b200._lib import Sph3Error
    ic = _state()
    ctx = _ctx(ic)
    for rows in ((-1, 5), (5, 4), (0, N + 1)):
        with pytest.raises(Sph3Error):
            ctx.compute("density", rows=rows)
    ctx.compute("density", rows=(7, 7))  # empty slice: nothing to do
    ctx.close()


def test_mpi_drop_in_slices_match_full():
    from sph_3_b200 import libsx
    ic = _state(9)
    pos, m = ic["pos"], ic["m"]
    h = libsx.do_smoothingX((pos, pos))
    h = libsx.h_smooth_fast(pos, h)
    rho = libsx.getDensity(pos, m, h)
    parts = [(0, 6000), (6000, 13000), (13000, N)]
    got = np.concatenate([libsx.getDensity_mpi(a, b, pos, m, h) for a, b in parts])
    assert np.array_equal(got, rho)
    hs = np.concatenate([libsx.h_smooth_fast_mpi(a, b, pos, h) for a, b in parts])
    assert np.array_equal(hs, libsx.h_smooth_fast(pos, h))
