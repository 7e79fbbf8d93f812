"""Batched ensembles: many independent Evrard clouds stepped in one launch
per pass must give what separate runs of each cloud give."""
import numpy as np
import pytest

from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _batch_ic(ncloud=6, seed=5):
    from sph_3_b200.ic import evrard_batch
    return evrard_batch(ncloud=ncloud, seed=seed, n_min=1500, n_max=6000)


def test_batch_fp64_exact_gravity_matches_single_runs():
    from sph_3_b200 import Config, Context
    b = _batch_ic()
    cfg = Config(precision="fp64", theta=0.0, h_mode="refstep", n_ngb=64, h_max_iter=4000)
    ctx = Context(cfg)
    ctx.set_clouds(b["counts"])
    ctx.set_particles(b["pos"], b["m"], vel=b["vel"], u=b["u"])
    ctx.first_step(1e-3)
    ctx.step(1e-3, 2)
    assert ctx.status() == 0, ctx.status_names()
    got = {k: ctx.get_field(k) for k in ("pos", "rho", "u", "h")}
    ctx.close()
    beg = 0
    for k, cnt in enumerate(b["counts"]):
        sl = slice(beg, beg + cnt)
        one = Context(cfg)
        one.set_particles(b["pos"][sl], b["m"][sl], vel=b["vel"][sl], u=b["u"][sl])
        one.first_step(1e-3)
        one.step(1e-3, 2)
        for f in got:
            assert rel_err(got[f][sl], one.get_field(f)) < 1e-9, (k, f)
        one.close()
        beg += cnt


def test_batch_mixed_vs_per_cloud_fp64():
    """The batched mixed path against per-cloud plain-FP64 runs (theta = 0.5
    in both): positions after 2 steps within 1e-6 of each cloud's radius,
    densities within 1e-3 (the h windows settle slightly differently)."""
    from sph_3_b200 import Config, Context
    b = _batch_ic(ncloud=5, seed=9)
    ctx = Context(Config(precision="mixed"))
    ctx.set_clouds(b["counts"])
    ctx.set_particles(b["pos"], b["m"], vel=b["vel"], u=b["u"])
    ctx.first_step(1e-3)
    ctx.step(1e-3, 2)
    assert ctx.status() == 0, ctx.status_names()
    pos, rho = ctx.get_field("pos"), ctx.get_field("rho")
    ctx.close()
    beg = 0
    for k, cnt in enumerate(b["counts"]):
        sl = slice(beg, beg + cnt)
        one = Context(Config(precision="fp64"))
        one.set_particles(b["pos"][sl], b["m"][sl], vel=b["vel"][sl], u=b["u"][sl])
        one.first_step(1e-3)
        one.step(1e-3, 2)
        assert np.abs(pos[sl] - one.get_field("pos")).max() < 1e-6 * b["R"][k]
        assert np.median(np.abs(rho[sl] / one.get_field("rho") - 1.0)) < 1e-3
        one.close()
        beg += cnt


def test_batch_of_256_clouds_runs_and_conserves_mass():
    from sph_3_b200 import Config, Context
    from sph_3_b200.ic import evrard_batch
    b = evrard_batch(ncloud=256, seed=1, n_min=256, n_max=2048)
    ctx = Context(Config(precision="mixed"))
    ctx.set_clouds(b["counts"])
    ctx.set_particles(b["pos"], b["m"], vel=b["vel"], u=b["u"])
    ctx.first_step(1e-3)
    ctx.step(1e-3, 3)
    assert ctx.status() == 0, ctx.status_names()
    e = ctx.energy()
    assert abs(e["M"] - b["M"].sum()) < 1e-9 * b["M"].sum()
    ctx.close()
