"""The C oracle against the golden vectors produced by the reference's own
numba functions (tests/golden/make_golden.py).  Bit-exact everywhere: same
operation order, no FMA contraction, numba's integer-power expansion."""
import numpy as np
import pytest

CASES = ["evrard600", "evrard1500"]


@pytest.mark.parametrize("name", CASES)
def test_h_bootstrap_and_search_bitexact(oc, golden, name):
    g = golden(name)
    pos, n = g["pos"], g["pos"].shape[0]
    assert np.array_equal(oc.smoothing_length_mpi(0, n, pos), g["h0"])
    assert np.array_equal(oc.do_smoothingX((pos, pos)), g["h0"])
    assert np.array_equal(oc.h_smooth_fast(pos, g["h0"]), g["h"])
    b, e = g["h_from_pert_range"]
    assert np.array_equal(oc.h_smooth_fast_mpi(b, e, pos, g["h_pert"]), g["h_from_pert"])


@pytest.mark.parametrize("name", CASES)
def test_density_bitexact(oc, golden, name):
    g = golden(name)
    assert np.array_equal(oc.getDensity(g["pos"], g["m"], g["h"]), g["rho"])
    b, e = g["rho_mpi_range"]
    assert np.array_equal(oc.getDensity_mpi(b, e, g["pos"], g["m"], g["h"]), g["rho_mpi"])


@pytest.mark.parametrize("name", CASES)
def test_hydro_bitexact(oc, golden, name):
    g = golden(name)
    gama, alpha, beta, eta, G = g["consts"]
    a = (g["pos"], g["vel"], g["rho"], g["P"], g["c"], g["h"], g["m"])
    n = g["pos"].shape[0]
    assert np.array_equal(oc.getAcc_sph(*a, gama, eta, alpha, beta), g["acc_sph"])
    assert np.array_equal(oc.get_dU(*a, gama, eta, alpha, beta), g["dudt"])
    assert np.array_equal(oc.getAcc_sph_mpiXXX(0, n, *a, gama, eta, alpha, beta), g["acc_mg"])
    assert np.array_equal(oc.get_dU_mpiXXXX(0, n, *a, gama, eta, alpha, beta), g["dudt_mg"])
    dv, cv = oc.div_curlVel(g["pos"], g["vel"], g["rho"], g["m"], g["h"])
    assert np.array_equal(dv, g["divV"]) and np.array_equal(cv, g["curlV"])
    assert np.array_equal(oc.getAcc_sph_shear(*a, g["divV"], g["curlV"], alpha), g["acc_sh"])
    assert np.array_equal(oc.get_dU_shear(*a, g["divV"], g["curlV"], alpha), g["dudt_sh"])


@pytest.mark.parametrize("name", CASES)
def test_gravity_energy_bitexact(oc, golden, name):
    g = golden(name)
    G = g["consts"][4]
    n = g["pos"].shape[0]
    assert np.array_equal(oc.getAcc_g_smth_mpi(0, n, g["pos"], g["m"], G, g["eps"]), g["acc_g"])
    assert np.array_equal(oc.getAcc_g_smth(g["pos"], g["m"], G, g["eps"]), g["acc_g_sym"])
    assert oc.getKE(g["vel"], g["m"]) == float(g["KE"])
    assert oc.getPE(g["pos"], g["m"], G, g["eps"]) == float(g["PE"])


def test_edge_cases(oc, golden):
    g = golden("coincident120")
    gama, alpha, beta, eta, G = g["consts"]
    assert np.array_equal(oc.getDensity(g["pos"], g["m"], g["h"]), g["rho"])
    a = (g["pos"], g["vel"], g["rho"], g["P"], g["c"], g["h"], g["m"])
    assert np.array_equal(oc.getAcc_sph(*a, gama, eta, alpha, beta), g["acc_sph"])
    assert np.array_equal(oc.get_dU(*a, gama, eta, alpha, beta), g["dudt"])
    s = golden("single")
    assert np.array_equal(oc.getDensity(s["pos"], s["m"], s["h"]), s["rho"])


def test_empty_input(oc):
    pos = np.zeros((0, 3))
    assert oc.getDensity(pos, np.zeros(0), np.zeros(0)).shape == (0,)
    assert oc.getAcc_g_smth_mpi(0, 0, pos, np.zeros(0), 1.0, np.zeros(0)).shape == (0, 3)


def test_thread_count_independent(oc, golden):
    g = golden("evrard600")
    nt = oc.num_threads()
    oc.set_threads(1)
    try:
        r1 = oc.getDensity(g["pos"], g["m"], g["h"])
    finally:
        oc.set_threads(nt)
    assert np.array_equal(r1, g["rho"])


def test_rows_form_matches_full(oc, golden):
    g = golden("evrard1500")
    rows = np.array([0, 17, 1499, 800, 3])
    full = oc.getDensity(g["pos"], g["m"], g["h"])
    assert np.array_equal(oc.density_rows(g["pos"], g["m"], g["h"], rows), full[rows])
    nb = oc.neighbours(g["pos"], g["h"], 17)
    d = np.linalg.norm(g["pos"] - g["pos"][17], axis=1)
    q = d / (0.5 * (g["h"][17] + g["h"]))
    assert set(nb.tolist()) == set(np.nonzero(q <= 2.0)[0].tolist())


def test_h_cap_flags(oc, golden):
    g = golden("evrard600")
    h, st = oc.h_smooth_rows(g["pos"], g["h0"] * 3.0, rows=np.arange(10), max_iter=3)
    assert np.all(st == -1)


def test_gravity_forms_bitexact(oc, golden):
    """Every gravity form (unequal masses and softening lengths), the mimj
    partial arrays of a three-way partition, getPE and do_smoothingX with
    distinct query points (sph_code/libsx.py:583-747, 752-774, 908-947)."""
    g = golden("grav_forms")
    pos, m, eps, G = g["pos"], g["m"], g["eps"], float(g["G"])
    assert np.array_equal(oc.getAcc_g_smth(pos, m, G, eps), g["acc_sym"])
    assert np.array_equal(oc.getAcc_g_smthx(pos, m, G, eps), g["acc_x"])
    b, e = g["acc_rows_range"]
    assert np.array_equal(oc.getAcc_g_smth_mpi(b, e, pos, m, G, eps), g["acc_rows"])
    for k, (b, e) in enumerate(g["mimj_parts"]):
        assert np.array_equal(oc.getAcc_g_smth_mimj_mpi(b, e, pos, m, G, eps), g["mimj"][k])
    assert oc.getPE(pos, m, G, eps) == float(g["PE"])
    assert np.array_equal(oc.do_smoothingX((pos, g["q"])), g["hq"])
    # the three full forms agree bit for bit, and the partials sum to the field
    assert np.array_equal(g["acc_sym"], g["acc_x"])
    assert np.allclose(g["mimj"].sum(axis=0), g["acc_sym"], rtol=1e-12, atol=1e-12 * np.abs(g["acc_sym"]).max())


def test_timestep_oracle_vs_reference_kernel(oc, golden):
    """The oracle's FP64 restatement of the time-step criterion against the
    reference's own GPU kernel dt_array_indiv_dt (float32, run unchanged by
    tests/golden/make_timestep.py) on the same float32-exact inputs:
    relative 1e-6 (measured 1.8e-7: the float32 kernel's rounding)."""
    g = golden("timestep_ref")
    dt, dh = oc.timestep_rows(g["pos"], g["vel"], g["acc_tot"], g["acc_g"], g["h"], g["c"], g["divV"], g["eps"],
                              float(g["c_cfl"]), float(g["alpha"]))
    ref = g["dt"].astype(np.float64)
    assert np.max(np.abs(dt - ref) / ref) < 1e-6
    dref = g["dhdt"].astype(np.float64)
    assert np.max(np.abs(dh - dref)) < 1e-6 * np.max(np.abs(dref))
