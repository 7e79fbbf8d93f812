"""The Evrard N = 10,000 configuration the reference runs on its CPU, checked
on every row: seed 0, M = R = G = 1, r = sqrt(U), isotropic directions, equal
masses, v = 0, u = 0.05, gamma = 5/3, N_ngb = 64, eps = 0.01, one full step
(start-up forces of sph_code/sph_serial.py:85-134, then one loop body of
:142-193), FP64.

* Exact gravity (theta = 0): the GPU step against the oracle's composition of
  the reference functions in the serial driver's order (oracle/step.py, the
  h bootstrap included): h bit for bit, positions, velocities, u and density
  to 1e-9, accelerations and du/dt to 1e-8.
* Barnes-Hut theta = 0.5 (the same step through the FP64 tree walk): gravity
  against the FP64 direct sum on all 10,000 rows, median relative error below
  1e-3 (p99 below 1e-2).
"""
import numpy as np
import pytest

from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

N = 10000
DT = 1e-3
PARAMS = dict(n_ngb=64, n_boot=50, gamma=5.0 / 3.0, alpha=1.0, beta=2.0, eta=0.1, G=1.0)


@pytest.fixture(scope="module")
def ic():
    from sph_3_b200.ic import evrard
    d = evrard(N, seed=0)
    d["eps"] = np.full(N, 0.01)
    return d


def _gpu_step(ic, theta):
    from sph_3_b200 import Config, Context
    ctx = Context(Config(precision="fp64", h_mode="refstep", n_ngb=64, n_boot=50, theta=theta,
                         h_max_iter=4000, use_graph=True))
    # no h given: the start-up bootstraps it (half the 51st-nearest distance)
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=ic["eps"])
    ctx.first_step(DT)
    ctx.step(DT, 1)
    got = {k: ctx.get_field(k) for k in ("pos", "vel", "u", "h", "rho", "acc", "acc_g", "dudt")}
    status = ctx.status()
    ctx.close()
    return got, status


def test_evrard10k_fp64_step_all_rows(ic, oc):
    from oracle.step import serial_first_step, serial_step
    st = dict(pos=ic["pos"], vel=ic["vel"], m=ic["m"], u=ic["u"], eps=ic["eps"], h=None)
    ref = serial_step(oc, serial_first_step(oc, st, DT, PARAMS), DT, PARAMS)
    got, status = _gpu_step(ic, 0.0)
    assert status == 0
    assert np.array_equal(got["h"], ref["h"])
    for k in ("pos", "vel", "u", "rho"):
        assert rel_err(got[k], ref[k]) < 1e-9, k
    assert rel_err(got["acc"], ref["acc"], floor_frac=1e-3) < 1e-8
    assert rel_err(got["dudt"], ref["dudt"], floor_frac=1e-3) < 1e-8
    cnt = oc.count_within(got["pos"], got["h"])
    assert np.all((cnt >= 59) & (cnt <= 69))


def test_evrard10k_bh_gravity_vs_direct_sum(ic, oc):
    got, status = _gpu_step(ic, 0.5)
    assert status == 0
    ref = oc.grav_direct_rows(got["pos"], ic["m"], 1.0, ic["eps"])
    err = np.linalg.norm(got["acc_g"] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    print("Evrard 10k, BH theta=0.5 vs FP64 direct sum on all rows: median %.2e p95 %.2e p99 %.2e max %.2e"
          % (np.median(err), np.percentile(err, 95), np.percentile(err, 99), err.max()))
    assert np.median(err) < 1e-3
    assert np.percentile(err, 99) < 1e-2
