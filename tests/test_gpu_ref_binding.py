"""The ctypes binding a maintainer drops into the reference's sph_code/
(sph_3_b200/ref_binding.py) gives the reference's
getDensity and getAcc_g_smth results: checked against the oracle (which is
pinned to the reference's own outputs) on a seeded Evrard set."""
import numpy as np
import pytest

from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def test_ref_binding_density_and_gravity(oc):
    from sph_3_b200 import ref_binding as rb
    from sph_3_b200.ic import evrard
    ic = evrard(3000, seed=5)
    pos, m = ic["pos"], ic["m"]
    h = oc.smoothing_length_rows(pos, k=50)
    rho = rb.getDensity(pos, m, h)
    assert rel_err(rho, oc.density_rows(pos, m, h, np.arange(len(m)))) < 1e-10
    acc = rb.getAcc_g_smth(pos, m, 1.0, 0.01)
    ref = oc.grav_direct_rows(pos, m, 1.0, np.full(len(m), 0.01), np.arange(len(m)))
    assert np.array_equal(acc, ref)
