"""Per-particle time step (the reference's dt_array_indiv_dt,
Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:
1189-1262) against the oracle's restatement, in both signal-velocity modes:
over every particle of the system (the reference's loop) and over the hydro
pairs |r_ij| <= h_i + h_j."""
import numpy as np
import pytest

from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _state(prec, n=3000, seed=21):
    from sph_3_b200 import Config, Context
    from sph_3_b200.ic import evrard
    ic = evrard(n, seed=seed)
    ic["vel"] = np.random.default_rng(seed).normal(scale=0.2, size=(n, 3))
    ctx = Context(Config(precision=prec, eps=0.01))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=np.full(n, 0.01))
    ctx.compute("boot_h", "h", "density", "gravity", "acc_sph", "dudt")
    assert ctx.status() == 0, ctx.status_names()
    return ctx


def _oracle(oc, ctx, neighbours):
    f = {k: ctx.get_field(k) for k in ("pos", "vel", "acc", "acc_g", "h", "c", "divV", "eps")}
    return oc.timestep_rows(f["pos"], f["vel"], f["acc"], f["acc_g"], f["h"], f["c"], f["divV"], f["eps"],
                            0.25, 1.0, neighbours=neighbours)


@pytest.mark.parametrize("all_pairs", [True, False])
def test_timestep_fp64_matches_oracle(oc, all_pairs):
    ctx = _state("fp64")
    dt, dt_min = ctx.timestep(0.25, all_pairs=all_pairs)
    ref, dh_ref = _oracle(oc, ctx, neighbours=not all_pairs)
    assert rel_err(dt, ref) < 1e-10
    assert rel_err(ctx.get_field("dhdt"), dh_ref, floor_frac=1e-6) < 1e-10
    assert dt_min == pytest.approx(dt.min(), rel=0, abs=0)
    assert np.all(np.isfinite(dt)) and np.all(dt > 0)
    ctx.close()


def test_timestep_mixed_close_to_fp64_oracle(oc):
    ctx = _state("mixed")
    dt, dt_min = ctx.timestep(0.25, all_pairs=False)
    ref, _ = _oracle(oc, ctx, neighbours=True)
    assert rel_err(dt, ref) < 1e-4
    assert dt_min == dt.min()
    ctx.close()


def test_neighbour_max_is_bounded_by_all_pairs_max(oc):
    """the all-pairs maximum can only be larger, so its dt only smaller"""
    ctx = _state("fp64")
    dt_n, _ = ctx.timestep(0.25, all_pairs=False)
    dt_a, _ = ctx.timestep(0.25, all_pairs=True)
    assert np.all(dt_a <= dt_n * (1 + 1e-12))
    ctx.close()


def test_timestep_vs_reference_kernel_golden(golden):
    """sph3_timestep over every particle (the reference's loop) against the
    reference's own float32 GPU kernel on the same float32-exact state
    (tests/golden/timestep_ref.npz): relative 1e-5; div v is recomputed here
    from the positions and velocities (FP64), the kernel took it rounded."""
    from sph_3_b200 import Config, Context
    g = golden("timestep_ref")
    ctx = Context(Config(precision="fp64", eps=0.01))
    ctx.set_particles(g["pos"], g["m"], vel=g["vel"], u=g["u"], h=g["h"], eps=g["eps"])
    ctx.set_field("rho", g["rho"])
    ctx.set_field("c", g["c"])
    ctx.set_field("acc", g["acc_tot"])
    ctx.set_field("acc_g", g["acc_g"])
    dt, dt_min = ctx.timestep(float(g["c_cfl"]), all_pairs=True)
    ref = g["dt"].astype(np.float64)
    err = np.abs(dt - ref) / ref
    print("time step vs the reference kernel: max rel %.2e" % err.max())
    assert err.max() < 1e-5
    assert dt_min == pytest.approx(ref.min(), rel=1e-5)
    dh = ctx.get_field("dhdt")
    dref = g["dhdt"].astype(np.float64)
    assert np.max(np.abs(dh - dref)) < 1e-5 * np.max(np.abs(dref))
    ctx.close()
