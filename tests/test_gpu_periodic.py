"""Periodic boxes (the Sedov and Kelvin-Helmholtz workloads): minimum-image
parity with the oracle, hydro only.  The reference CPU code has no periodic
support (its GPU driver only wraps positions, KH/hfvCLibs_v7_hfv_v8.2.h:
1125-1157), so the oracle adds the minimum image to the reference formulas."""
import numpy as np
import pytest

from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _ctx(prec, box, **kw):
    from sph_3_b200 import Config, Context
    return Context(Config(precision=prec, gravity=False, box=box, **kw))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 2e-5)])
def test_sedov_lattice_density_and_hydro(oc, prec, tol):
    from sph_3_b200.ic import sedov
    ic = sedov(n_side=16, seed=3)
    box = ic["box"]
    ctx = _ctx(prec, box)
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h", "h", "density")
    assert ctx.status() == 0, ctx.status_names()
    h, rho = ctx.get_field("h"), ctx.get_field("rho")
    n = ic["pos"].shape[0]
    rows = np.arange(0, n, 7)
    rho_ref = oc.density_rows(ic["pos"], ic["m"], h, rows, box=box)
    assert rel_err(rho[rows], rho_ref) < tol
    cnt = oc.count_within(ic["pos"], h, rows, box=box)
    assert np.all((cnt >= 59) & (cnt <= 69))
    vel = np.random.default_rng(0).normal(scale=0.2, size=(n, 3))
    ctx.set_field("vel", vel)
    ctx.compute("acc_sph", "dudt")
    P, c = ctx.get_field("P"), ctx.get_field("c")
    a_ref, du_ref = oc.hydro_rows(ic["pos"], vel, rho, P, c, h, ic["m"], 0, 1.0, 2.0, 0.1, rows=rows, box=box)
    assert rel_err(ctx.get_field("acc_sph")[rows], a_ref, floor_frac=1e-2) < 100 * tol
    assert rel_err(ctx.get_field("dudt")[rows], du_ref, floor_frac=1e-2) < 100 * tol
    ctx.close()


def test_sedov_steps_fp64_match_oracle(oc):
    """Five steps of dt = 1e-4 after the blast deposit, reference h rule
    (N_ngb = 64), FP64 path vs the oracle's serial-driver composition."""
    from oracle.step import serial_first_step, serial_step
    from sph_3_b200.ic import sedov
    ic = sedov(n_side=12, seed=4)
    box = ic["box"]
    dt = 1e-4
    params = dict(n_ngb=64, gravity=False, box=box)
    h0 = oc.smoothing_length_rows(ic["pos"], k=50, box=box)
    st = dict(pos=ic["pos"], vel=ic["vel"], m=ic["m"], u=ic["u"], eps=np.full(len(ic["m"]), 0.01), h=h0)
    ref = serial_first_step(oc, st, dt, params)
    for _ in range(5):
        ref = serial_step(oc, ref, dt, params)
    ctx = _ctx("fp64", box, h_mode="refstep", n_ngb=64, h_max_iter=4000)
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], h=h0)
    ctx.first_step(dt)
    ctx.step(dt, 5)
    assert ctx.status() == 0, ctx.status_names()
    d = np.abs(ctx.get_field("pos") - ref["pos"])
    d = np.minimum(d, 1.0 - d)  # periodic distance
    assert d.max() < 1e-10
    assert rel_err(ctx.get_field("u"), ref["u"]) < 1e-8
    assert rel_err(ctx.get_field("rho"), ref["rho"]) < 1e-8
    ctx.close()


def test_thin_box_is_flagged():
    """A slab thinner than the kernel support has no unique minimum image."""
    from sph_3_b200 import STATUS_BITS
    from sph_3_b200.ic import kelvin_helmholtz
    ic = kelvin_helmholtz(n=6000, seed=2)
    ctx = _ctx("mixed", ic["box"])
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h", "h")
    assert ctx.status() & STATUS_BITS["BOX_TOO_SMALL"]
    ctx.close()


def test_kelvin_helmholtz_slab_density(oc):
    from sph_3_b200.ic import kelvin_helmholtz
    ic = kelvin_helmholtz(n=200000, seed=2)
    box = ic["box"]
    ctx = _ctx("mixed", box)
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h", "h", "density")
    assert ctx.status() == 0, ctx.status_names()
    h, rho = ctx.get_field("h"), ctx.get_field("rho")
    rows = np.arange(0, ic["pos"].shape[0], 97)
    assert rel_err(rho[rows], oc.density_rows(ic["pos"], ic["m"], h, rows, box=box)) < 2e-5
    inner = np.abs(ic["pos"][:, 1] - 0.5) < 0.2
    outer = np.abs(ic["pos"][:, 1] - 0.5) > 0.3
    assert 1.7 < np.median(rho[inner]) < 2.3 and 0.85 < np.median(rho[outer]) < 1.15
    ctx.step(1e-4, 3)
    assert ctx.status() == 0
    p = ctx.get_field("pos")
    assert p.min() >= 0.0 and p[:, 0].max() < 1.0 and p[:, 2].max() < 1.0 / 16.0
    ctx.close()
