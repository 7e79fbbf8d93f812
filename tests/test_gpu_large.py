"""Evrard N = 1,048,576 (the benchmark workload): errors of the mixed path
against FP64 references, stated per quantity, on sampled rows.

* gravity: Barnes-Hut theta = 0.5 against the FP64 direct sum on 4,096
  random particles (median relative error < 1e-3, p95/p99 printed); the GPU
  direct sum itself is checked against the CPU oracle on 64 rows;
* density: against the oracle at the GPU's own h, rel < 1e-5 (mixed) and
  < 1e-10 (FP64 path);
* h: the exact oracle count N(r < 2h) lies in 64 +- 5 for every sampled row;
* hydro: acceleration and du/dt against the oracle (vector relative error,
  median < 1e-5, max < 1e-3 mixed; 1e-9 FP64);
* energy: |dE/E| over 100 KDK steps of dt = 1e-3 (mixed) below 1e-3.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 1048576


@pytest.fixture(scope="module")
def ic():
    from sph_3_b200.ic import evrard
    d = evrard(N, seed=0)
    d["eps"] = np.full(N, 0.01)
    return d


def _vec_err(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def test_gravity_bh_vs_fp64_direct(ic, oc):
    from sph_3_b200 import Config, Context
    ctx = Context(Config(precision="mixed", theta=0.5))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=ic["eps"])
    ctx.compute("gravity")
    rows = np.random.default_rng(0).choice(N, 4096, replace=False)
    acc = ctx.get_field("acc_g")[rows]
    ref, _ = ctx.gravity_direct_rows(rows)
    err = _vec_err(acc, ref)
    print("BH theta=0.5 vs FP64 direct: median %.3e p95 %.3e p99 %.3e max %.3e"
          % (np.median(err), np.percentile(err, 95), np.percentile(err, 99), err.max()))
    assert np.median(err) < 1e-3
    assert np.percentile(err, 99) < 1e-2
    cpu = oc.grav_direct_rows(ic["pos"], ic["m"], 1.0, ic["eps"], rows[:64])
    assert np.max(_vec_err(ref[:64], cpu)) < 1e-10
    ctx.close()


@pytest.mark.parametrize("prec,tol_rho,tol_acc_med,tol_acc_max", [("mixed", 1e-5, 1e-5, 1e-3),
                                                                  ("fp64", 1e-10, 1e-9, 1e-9)])
def test_sph_first_step_vs_oracle(ic, oc, prec, tol_rho, tol_acc_med, tol_acc_max):
    from sph_3_b200 import Config, Context
    ctx = Context(Config(precision=prec))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=ic["eps"])
    ctx.compute("boot_h", "h", "density")
    assert ctx.status() == 0, ctx.status_names()
    h = ctx.get_field("h")
    rho = ctx.get_field("rho")
    rng = np.random.default_rng(1)
    rows = rng.choice(N, 384, replace=False)
    rho_ref = oc.density_rows(ic["pos"], ic["m"], h, rows)
    assert np.max(np.abs(rho[rows] - rho_ref) / rho_ref) < tol_rho
    cnt = oc.count_within(ic["pos"], h, rows)
    assert np.all((cnt >= 59) & (cnt <= 69)), (cnt.min(), cnt.max())
    # hydro with a random velocity field so that the viscosity is exercised
    vel = rng.normal(scale=0.1, size=(N, 3))
    ctx.set_field("vel", vel)
    ctx.compute("acc_sph", "dudt")
    acc = ctx.get_field("acc_sph")
    du = ctx.get_field("dudt")
    P, c = ctx.get_field("P"), ctx.get_field("c")
    a_ref, du_ref = oc.hydro_rows(ic["pos"], vel, rho, P, c, h, ic["m"], 0, 1.0, 2.0, 0.1, rows=rows[:128])
    e = _vec_err(acc[rows[:128]], a_ref)
    print("%s hydro accel vs oracle: median %.2e max %.2e" % (prec, np.median(e), e.max()))
    assert np.median(e) < tol_acc_med and e.max() < tol_acc_max
    ed = np.abs(du[rows[:128]] - du_ref) / np.maximum(np.abs(du_ref), 1e-3 * np.sqrt(np.mean(du_ref ** 2)))
    assert np.median(ed) < tol_acc_med and ed.max() < 10 * tol_acc_max
    ctx.close()


def test_energy_drift_100_steps(ic):
    from sph_3_b200 import Config, Context
    ctx = Context(Config(precision="mixed"))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=ic["eps"])
    ctx.first_step(1e-3)
    e0 = ctx.energy()
    ctx.step(1e-3, 100)
    e1 = ctx.energy()
    drift = abs((e1["E"] - e0["E"]) / e0["E"])
    print("energy drift over 100 steps: %.3e (E0 %.6f, E1 %.6f)" % (drift, e0["E"], e1["E"]))
    assert ctx.status() == 0, ctx.status_names()
    assert drift < 1e-3
    assert abs(e1["px"]) + abs(e1["py"]) + abs(e1["pz"]) < 1e-4
    ctx.close()
