"""eps = h (the reference GPU driver's set_eps_of_gas_to_h,
Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:584-593):
after the h search the softening lengths equal the smoothing lengths, and
gravity (with the tree's softening moments refitted) matches the oracle's
direct sum with those softening lengths."""
import numpy as np
import pytest

from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,theta,tol", [("fp64", 0.0, 1e-10), ("mixed", 0.5, 1e-3)])
def test_eps_follows_h(oc, prec, theta, tol):
    from sph_3_b200 import Config, Context
    from sph_3_b200.ic import evrard
    n = 5000
    ic = evrard(n, seed=31)
    ctx = Context(Config(precision=prec, theta=theta, eps_from_h=True))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=np.full(n, 0.01))
    ctx.compute("boot_h", "h", "gravity")
    assert ctx.status() == 0, ctx.status_names()
    h, eps = ctx.get_field("h"), ctx.get_field("eps")
    assert np.array_equal(h, eps)
    acc = ctx.get_field("acc_g")
    ref = oc.grav_direct_rows(ic["pos"], ic["m"], 1.0, h, np.arange(n))
    if theta == 0.0:
        assert rel_err(acc, ref) < tol
    else:
        err = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert np.median(err) < tol
    # a step keeps eps = h with the new h
    ctx.first_step(1e-4)
    ctx.step(1e-4, 2)
    assert np.array_equal(ctx.get_field("h"), ctx.get_field("eps"))
    ctx.close()
