"""Failure detection without faulting the GPU: bad input and impossible
requests end in a status bit or an error code, never a trap or a hang."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_nan_position_sets_status_and_walks_skip():
    from sph_3_b200 import Config, Context, STATUS_BITS
    from sph_3_b200.ic import evrard
    ic = evrard(5000, seed=1)
    ic["pos"][17, 1] = np.nan
    ctx = Context(Config())
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.first_step(1e-3)
    ctx.step(1e-3, 2)
    s = ctx.status(clear=True)
    assert s & STATUS_BITS["NAN_INPUT"]
    ctx.close()


def test_h_search_that_cannot_converge_is_flagged():
    """A system with fewer particles than the lower edge of the window."""
    from sph_3_b200 import Config, Context, STATUS_BITS
    from sph_3_b200.ic import evrard
    ic = evrard(40, seed=2)
    ctx = Context(Config(h_max_iter=20))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h", "h")
    assert ctx.status() & STATUS_BITS["H_NOT_CONVERGED"]
    ctx.close()


def test_zero_density_flagged():
    from sph_3_b200 import Config, Context, STATUS_BITS
    from sph_3_b200.ic import evrard
    ic = evrard(2000, seed=3)
    ctx = Context(Config(gravity=False))
    ctx.set_particles(ic["pos"], np.zeros(2000), vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h", "h", "density")
    assert ctx.status() & STATUS_BITS["ZERO_DENSITY"]
    ctx.close()


def test_tiny_and_empty_systems():
    from sph_3_b200 import Config, Context
    ctx = Context(Config())
    ctx.set_particles(np.zeros((0, 3)), np.zeros(0))
    ctx.first_step(1e-3)
    ctx.step(1e-3, 1)
    assert ctx.get_field("rho").shape == (0,)
    ctx.set_particles(np.array([[0.3, -0.1, 0.2]]), np.array([2.0]), h=np.array([0.1]))
    ctx.compute("density")
    # mixed path: FP32 kernel arithmetic
    assert abs(ctx.get_field("rho")[0] / (2.0 / np.pi / 0.1 ** 3) - 1.0) < 1e-6
    ctx.close()


def test_bad_arguments_raise():
    from sph_3_b200 import Config, Context, Sph3Error
    ctx = Context(Config())
    with pytest.raises(Sph3Error):
        ctx.get_field("rho")  # nothing loaded
    ctx.set_particles(np.random.default_rng(0).random((100, 3)), np.full(100, 0.01))
    with pytest.raises(Sph3Error):
        ctx.get_field("rho", rows=(50, 200))
    with pytest.raises(Sph3Error):
        ctx.set_config(Config(leaf_size=0))
    ctx.close()
    with pytest.raises(Sph3Error):
        Context(Config(box=(1.0, 1.0, 1.0), gravity=True))


def test_status_persists_until_cleared():
    from sph_3_b200 import Config, Context, STATUS_BITS
    from sph_3_b200.ic import evrard
    ic = evrard(30, seed=4)
    ctx = Context(Config(h_max_iter=5))
    ctx.set_particles(ic["pos"], ic["m"])
    ctx.compute("boot_h", "h")
    assert ctx.status(clear=True) & STATUS_BITS["H_NOT_CONVERGED"]
    assert ctx.status() == 0
    ctx.close()
