"""Heating/cooling step on the GPU (hcoolingZ,
Particles_in_BH_Tree_III/Evrard_Collapse_2024/hfvCLibs_v7_hfv_v8.1.h:1433-1623)
through the C ABI: the raw-array entry point against the reference kernel's
own outputs and the oracle, the linear-scan path of tables whose grids are
not ordered, and the cooled step of a context (after the u update, inside the
captured step graph) against the oracle applied to the uncooled step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EVRARD_UNITS = dict(unit_density_cgs=1e-24, unit_time_s=3e13, unit_u_cgs=1e12, unit_length_cm=3.086e21)


def _units(cooling, g):
    d, t, u, l, k = (float(x) for x in g["units"])
    return cooling.Units(unit_density_cgs=d, unit_time_s=t, unit_u_cgs=u, unit_length_cm=l, kpc_cm=k, z_index=1)


def test_raw_entry_matches_reference_and_oracle(oc, golden):
    from sph_3_b200 import cooling
    g = golden("cooling_ref")
    tab = cooling.CoolTable(g, device=0)
    assert tab.monotone() == (True, True, True, True)
    units = _units(cooling, g)
    u, ion = cooling.hcooling(tab, units, float(g["dt"]), g["u"], g["rho"], g["pos"], typ=g["typ"])
    gas = g["typ"] == 0
    # non-gas particles untouched, and so are their ion-fraction rows
    assert np.array_equal(u[~gas], g["u"][~gas])
    # the reference kernel's own outputs: the same table indices everywhere
    # and the same u, bit for bit
    assert np.array_equal(ion[gas], g["ionfrac"][gas])
    assert np.array_equal(u, g["u_new"])
    # the oracle (the same FP32 operations): bit for bit
    uo, io = oc.hcooling(g, g["units"], g["dt"], g["u"], g["rho"], g["pos"], typ=g["typ"])
    assert np.array_equal(u, uo)
    assert np.array_equal(ion[gas], io[gas])
    tab.close()


def test_torch_tensors_in_place_and_two_calls(oc, golden):
    import torch
    from sph_3_b200 import cooling
    g = golden("cooling_ref")
    tab = cooling.CoolTable(g, device=0)
    units = _units(cooling, g)
    dev = torch.device("cuda", 0)
    u = torch.tensor(g["u"], device=dev)
    rho = torch.tensor(g["rho"], device=dev)
    pos = torch.tensor(g["pos"], device=dev)
    typ = torch.tensor(g["typ"], device=dev)
    _, ion1 = cooling.hcooling(tab, units, float(g["dt"]), u, rho, pos, typ=typ)
    first = u.cpu().numpy()
    # a second call cools the already cooled u (the oracle does the same)
    _, ion2 = cooling.hcooling(tab, units, float(g["dt"]), u, rho, pos, typ=typ)
    torch.cuda.synchronize()
    uo1, _ = oc.hcooling(g, g["units"], g["dt"], g["u"], g["rho"], g["pos"], typ=g["typ"])
    uo2, io2 = oc.hcooling(g, g["units"], g["dt"], uo1, g["rho"], g["pos"], typ=g["typ"])
    assert np.array_equal(first, uo1)
    assert np.array_equal(u.cpu().numpy(), uo2)
    gas = g["typ"] == 0
    assert np.array_equal(ion2.cpu().numpy()[gas], io2[gas])
    tab.close()


def test_unordered_grids_use_the_linear_scan(oc):
    from sph_3_b200 import cooling
    rng = np.random.default_rng(11)
    tab = cooling.seeded_table(seed=4, dims=(9, 16, 12, 3, 5, 6))
    # unordered kpc grid and one non-monotone u column: the reference's
    # first-match scan, not a bisection
    tab["kpc"] = rng.permutation(tab["kpc"]).astype(np.float32)
    tab["uArr"][2, :, 3, 1] = rng.permutation(tab["uArr"][2, :, 3, 1])
    t = cooling.CoolTable(tab, device=0)
    assert t.monotone() == (False, True, True, False)
    n = 20000
    pos = rng.uniform(-2.5, 2.5, (n, 3)).astype(np.float32)
    units = cooling.Units(unit_density_cgs=1e-24, unit_time_s=3e13, unit_u_cgs=1e12, unit_length_cm=3.086e21)
    rho = (10.0 ** rng.uniform(-5, 5, n)).astype(np.float32)
    u = (10.0 ** rng.uniform(-4, 5, n)).astype(np.float32)
    for dt in (0.0, 1e-4, 3e-3, 1.0):
        ug, ig = cooling.hcooling(t, units, dt, u, rho, pos)
        uo, io = oc.hcooling(tab, units.as_tuple(), dt, u, rho, pos)
        assert np.array_equal(ug, uo), dt
        assert np.array_equal(ig, io), dt
    t.close()


def test_argument_checks():
    import ctypes
    from sph_3_b200 import _lib, cooling
    lib = _lib.load()
    tab = cooling.CoolTable(cooling.seeded_table(seed=2, dims=(3, 5, 4, 2, 2, 3)), device=0)
    bad = _lib.CoolUnits(1.0, 1.0, 1.0, 1.0, 1.0, 2)  # z_index past N_Z = 2
    f = ctypes.c_void_p(0)
    assert lib.sph3_hcooling(tab.handle, ctypes.byref(bad), ctypes.c_float(1.0), 0, None, f, f, f, f, f, None,
                             None, None) == _lib.C["SPH3_ERR_INVALID_ARG"]
    ok = _lib.CoolUnits(1.0, 1.0, 1.0, 1.0, 1.0, 1)
    assert lib.sph3_hcooling(tab.handle, ctypes.byref(ok), ctypes.c_float(1.0), 0, None, f, f, f, f, f, None,
                             None, None) == 0  # n = 0: nothing to do
    assert lib.sph3_hcooling(tab.handle, ctypes.byref(ok), ctypes.c_float(1.0), 4, None, None, f, f, f, f, None,
                             None, None) == _lib.C["SPH3_ERR_INVALID_ARG"]
    tab.close()


def _evrard_ctx(n, cool=None, units=None, use_graph=True):
    from sph_3_b200 import Config, Context
    from sph_3_b200.ic import evrard
    ic = evrard(n, seed=3)
    ctx = Context(Config(precision="mixed", use_graph=use_graph), device=0)
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=np.full(n, 0.01))
    if cool is not None:
        ctx.set_cooling(cool, units)
    return ctx


def test_context_step_cools_after_the_u_update(oc):
    from sph_3_b200 import cooling
    tab = cooling.seeded_table(seed=8, dims=(12, 40, 24, 3, 6, 12))
    t = cooling.CoolTable(tab, device=0)
    units = cooling.Units(**EVRARD_UNITS)
    n, dt = 8192, 1e-3
    plain = _evrard_ctx(n)
    cooled = _evrard_ctx(n, t, units)
    for c in (plain, cooled):
        c.first_step(dt)
    # one step each: identical until the cooling, which follows the u update
    plain.step(dt, 1)
    cooled.step(dt, 1)
    pos = plain.get_field("pos")
    rho = plain.get_field("rho")
    u0 = plain.get_field("u")
    assert np.array_equal(cooled.get_field("pos"), pos)
    assert np.array_equal(cooled.get_field("rho"), rho)
    uo, io = oc.hcooling(tab, units.as_tuple(), dt, u0.astype(np.float32), rho.astype(np.float32),
                         pos.astype(np.float32))
    uc = cooled.get_field("u")
    assert np.array_equal(uc, uo.astype(np.float64))
    assert np.array_equal(cooled.ionfrac(), io)
    assert np.mean(uc != u0) > 0.5  # the table did change u
    assert cooled.status() == 0, cooled.status_names()
    plain.close()
    cooled.close()
    t.close()


def test_context_cooling_in_the_step_graph_matches_eager():
    from sph_3_b200 import cooling
    tab = cooling.seeded_table(seed=9, dims=(12, 40, 24, 3, 6, 12))
    t = cooling.CoolTable(tab, device=0)
    units = cooling.Units(**EVRARD_UNITS)
    n, dt = 8192, 5e-4
    a = _evrard_ctx(n, t, units, use_graph=True)
    b = _evrard_ctx(n, t, units, use_graph=False)
    for c in (a, b):
        c.first_step(dt)
        c.step(dt, 5)  # the graph path captures after two warm steps
    for f in ("u", "pos", "vel", "rho", "h"):
        assert np.array_equal(a.get_field(f), b.get_field(f)), f
    assert np.array_equal(a.ionfrac(), b.ionfrac())
    assert a.kernels_per_step() > 0
    # cool_now once more on the current state, and cooling off again
    u_before = a.get_field("u")
    a.cool_now(dt)
    assert not np.array_equal(a.get_field("u"), u_before)
    a.set_cooling(None)
    with pytest.raises(RuntimeError):
        a.ionfrac()
    a.step(dt, 1)
    a.close()
    b.close()
    t.close()


@pytest.mark.parametrize("n_species,n", [(5, 19987), (16, 33), (17, 1001), (40, 4099)])
def test_ion_fraction_block_writes(oc, n_species, n):
    """Ragged warp blocks, species counts either side of the staged limit and
    non-gas rows, through the C ABI: gas rows equal the oracle's, non-gas rows
    keep the caller's contents."""
    import ctypes
    import torch
    from sph_3_b200 import _lib, cooling
    rng = np.random.default_rng(n_species * 1000 + n)
    tab = cooling.seeded_table(seed=n_species, dims=(5, 12, 9, 3, n_species, 7))
    t = cooling.CoolTable(tab, device=0)
    units = cooling.Units(unit_density_cgs=1e-24, unit_time_s=3e13, unit_u_cgs=1e12, unit_length_cm=3.086e21)
    pos = rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32)
    rho = (10.0 ** rng.uniform(-4, 4, n)).astype(np.float32)
    u = (10.0 ** rng.uniform(-3, 4, n)).astype(np.float32)
    typ = np.where(rng.random(n) < 0.2, 2, 0).astype(np.int32)
    dev = torch.device("cuda", 0)
    T = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    ud, rd, td = T(u), T(rho), T(typ)
    xs = [T(np.ascontiguousarray(pos[:, k])) for k in range(3)]
    ion = torch.full((n, n_species), -7.0, dtype=torch.float32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    cu = units.to_c()
    P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731
    lib = _lib.load()
    rc = lib.sph3_hcooling(t.handle, ctypes.byref(cu), ctypes.c_float(2e-3), n, P(td), P(ud), P(rd), P(xs[0]),
                           P(xs[1]), P(xs[2]), P(ion), P(status), None)
    assert rc == 0
    torch.cuda.synchronize()
    uo, io = oc.hcooling(tab, units.as_tuple(), 2e-3, u, rho, pos, typ=typ)
    gas = typ == 0
    got = ion.cpu().numpy()
    assert np.array_equal(ud.cpu().numpy(), uo)
    assert np.array_equal(got[gas], io[gas])
    assert np.all(got[~gas] == -7.0)
    t.close()
