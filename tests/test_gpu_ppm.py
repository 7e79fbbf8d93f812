"""Long-run physics check: the Evrard collapse at t = 0.8 against the 1-D PPM
solution the reference compares with (sph_code/ppm_profile/ppm1oaf, converted
to code units by tests/golden/make_ppm.py).  N = 262,144, mixed precision,
global time step from the reference's per-particle criterion.  Away from the
accretion shock (r ~ 0.15, which SPH smears over a few h) the binned profiles
follow PPM to a few per cent; the whole range [0.05, 0.8] is dominated by the
shock zone."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_evrard_t08_matches_ppm():
    from sph_3_b200 import Config, Context
    from sph_3_b200 import validate as V
    from sph_3_b200.ic import evrard
    d = np.load(os.path.join(HERE, "golden", "ppm_evrard.npz"))
    ppm = {k: d[k] for k in ("radius", "rho", "press", "vr")}
    n = 262144
    ic = evrard(n, seed=0)
    ctx = Context(Config(precision="mixed", n_ngb=64, eps=0.01))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=np.full(n, 0.01))
    t, steps, used = V.evolve(ctx, 0.8, dt_max=1e-3)
    assert abs(t - 0.8) < 1e-9 and min(used) >= 1e-3 / 64
    f = {k: ctx.get_field(k) for k in ("pos", "vel", "rho", "P", "m")}
    prof = V.radial_profile(f["pos"], f["vel"], f["rho"], f["P"], f["m"])
    whole = V.compare_ppm(prof, ppm, 0.05, 0.8)
    outer = V.compare_ppm(prof, ppm, 0.2, 0.8)
    core = V.compare_ppm(prof, ppm, 0.02, 0.1)
    print("steps %d, PPM errors: [0.05, 0.8] %s; [0.2, 0.8] %s; [0.02, 0.1] %s" % (steps, whole, outer, core))
    assert whole["rho"] < 0.2 and whole["vr"] < 0.1 and whole["press"] < 0.8
    assert outer["rho"] < 0.08 and outer["vr"] < 0.03 and outer["press"] < 0.2
    assert core["rho"] < 0.12 and core["vr"] < 0.01
    E = ctx.energy()
    assert np.isfinite(E["E"])
    ctx.close()
