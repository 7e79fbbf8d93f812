"""Heating/cooling step on the host: the oracle's FP32 restatement of the
reference's hcoolingZ (Particles_in_BH_Tree_III/Evrard_Collapse_2024/
hfvCLibs_v7_hfv_v8.1.h:1433-1623) against the reference kernel's own outputs
(tests/golden/cooling_ref.npz, made by tests/golden/make_cooling.py), the
table file layout of coolHeatGridJan2024.bin, and the C ABI's argument
checks (no GPU needed)."""
import ctypes

import numpy as np
import pytest

from sph_3_b200 import _lib, cooling


def test_oracle_matches_reference_kernel(oc, golden):
    g = golden("cooling_ref")
    u, ion = oc.hcooling(g, g["units"], g["dt"], g["u"], g["rho"], g["pos"], typ=g["typ"])
    gas = g["typ"] == 0
    # non-gas particles are left alone, with no ion fractions
    assert np.array_equal(u[~gas], g["u"][~gas])
    assert np.array_equal(g["u_new"][~gas], g["u"][~gas])
    assert not np.any(g["ionfrac"][~gas])
    # every table index agrees: the ion fractions are plain table reads
    assert np.array_equal(ion[gas], g["ionfrac"][gas])
    # u: the same FP32 operations, the interpolation fused as the reference
    # kernel's compiled form: bit for bit
    assert np.array_equal(u, g["u_new"])
    # the inputs reach every branch: below the first T row, interpolation,
    # above the last row, and radii / densities beyond both grids' ends
    uarr = g["uArr"]
    assert (g["u"][gas] * g["units"][2] < uarr.min()).any()
    assert (g["u"][gas] * g["units"][2] > uarr.max()).any()


def test_table_file_layout_round_trip(tmp_path):
    tab = cooling.seeded_table(seed=3, dims=(4, 6, 5, 3, 2, 7))
    p = tmp_path / "coolHeatGrid.bin"
    cooling.write_table(p, tab)
    raw = p.read_bytes()
    # header: N_kpc, N_T, N_nH, N_Z, N_M, N_t as int32, then the float arrays
    assert list(np.frombuffer(raw[:24], np.int32)) == [4, 6, 5, 3, 2, 7]
    n_float = 4 + 5 + 3 + 6 + 7 + 2 * (4 * 6 * 5 * 3 * 7) + 4 * 6 * 5 * 3 * 2 * 7 + 4 * 6 * 5 * 3
    assert len(raw) == 24 + 4 * n_float
    back = cooling.read_table(p)
    for k in ("kpc", "nH", "Z", "T", "t", "uEvol", "muArr", "metalz", "uArr"):
        assert np.array_equal(back[k], tab[k]), k
    # uArr is the last block, uEvol follows the five grids
    assert np.array_equal(np.frombuffer(raw[-4 * tab["uArr"].size:], np.float32), tab["uArr"].ravel())
    off = 24 + 4 * (4 + 5 + 3 + 6 + 7)
    assert np.array_equal(np.frombuffer(raw[off:off + 4 * tab["uEvol"].size], np.float32), tab["uEvol"].ravel())
    with pytest.raises(ValueError):
        (tmp_path / "short.bin").write_bytes(raw[:100])
        cooling.read_table(tmp_path / "short.bin")


def test_seeded_table_is_ordered():
    tab = cooling.seeded_table(seed=1)
    assert np.all(np.diff(tab["kpc"]) >= 0) and np.all(np.diff(tab["nH"]) > 0) and np.all(np.diff(tab["t"]) > 0)
    assert np.all(np.diff(tab["uArr"], axis=1) > 0)
    assert np.all(tab["uEvol"] > 0) and np.all((tab["metalz"] >= 0) & (tab["metalz"] <= 1))


def test_c_abi_argument_checks_without_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    bad = (ctypes.c_int32 * 6)(3, 4, 5, 0, 2, 3)
    f = (ctypes.c_float * 64)()
    assert lib.sph3_cool_table_create(0, bad, f, f, f, f, f, f, ctypes.byref(h)) == _lib.C["SPH3_ERR_INVALID_ARG"]
    assert lib.sph3_cool_table_create(0, None, f, f, f, f, f, f, ctypes.byref(h)) == _lib.C["SPH3_ERR_INVALID_ARG"]
    units = _lib.CoolUnits(1.0, 1.0, 1.0, 1.0, 1.0, 1)
    assert lib.sph3_hcooling(None, ctypes.byref(units), ctypes.c_float(1.0), 4, None, f, f, f, f, f, None, None,
                             None) == _lib.C["SPH3_ERR_INVALID_ARG"]
    assert lib.sph3_cool_table_destroy(None) == 0
    assert lib.sph3_set_cooling(None, None, None) == _lib.C["SPH3_ERR_INVALID_ARG"]


def test_units_layout_matches_header():
    # sph3_cool_units: five floats then an int32
    assert ctypes.sizeof(_lib.CoolUnits) == 24
    u = cooling.Units(1.5, 2.5, 3.5, 4.5, 5.5, 2).to_c()
    assert (u.unit_density_cgs, u.unit_time_s, u.unit_u_cgs, u.unit_length_cm, u.kpc_cm, u.z_index) == \
        (1.5, 2.5, 3.5, 4.5, 5.5, 2)
