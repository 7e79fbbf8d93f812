"""Neighbour lists of the mixed path: the density walk keeps each particle's
in-support pairs and the hydro pass runs over them; particles with more
neighbours than list_cap fall back to a walk.  All three routes (lists,
partial overflow, walk only) must give the same hydro results, and they must
match the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _err(a, b):
    """per-particle |a - b| / max(|b|, 1e-3 rms(b)) (vector norm for (N,3))"""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    if a.ndim == 1:
        a, b = a[:, None], b[:, None]
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.maximum(nb, 1e-3 * np.sqrt(np.mean(nb ** 2)))


def _hydro(ic, list_cap, visc="signal"):
    from sph_3_b200 import Config, Context
    ctx = Context(Config(precision="mixed", gravity=False, list_cap=list_cap, visc=visc))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h", "h", "density")
    if visc == "balsara":
        ctx.compute("divcurl")
    ctx.compute("acc_sph", "dudt")
    assert ctx.status() == 0, ctx.status_names()
    out = {k: ctx.get_field(k) for k in ("acc_sph", "dudt", "h", "rho", "P", "c", "nngb")}
    out["pairs"] = ctx.counters()["hydro_pairs"]
    ctx.close()
    return out


@pytest.mark.parametrize("visc", ["signal", "mg83", "balsara"])
def test_list_overflow_and_walk_agree(oc, visc):
    from sph_3_b200.ic import evrard
    ic = evrard(20000, seed=11)
    ic["vel"] = np.random.default_rng(3).normal(scale=0.3, size=ic["pos"].shape)
    full, part, walk = _hydro(ic, 128, visc), _hydro(ic, 64, visc), _hydro(ic, 0, visc)
    for k in ("h", "rho"):
        assert np.array_equal(full[k], walk[k])
    for name, other in (("partial", part), ("walk", walk)):
        for k in ("acc_sph", "dudt"):
            e = _err(other[k], full[k])
            print("%s %s vs lists: median %.2e max %.2e" % (name, k, np.median(e), e.max()))
            assert np.median(e) < 1e-6 and e.max() < 1e-4
    rows = np.arange(0, 20000, 97)
    v = {"signal": 0, "mg83": 1, "balsara": 2}[visc]
    if visc != "balsara":
        a_ref, du_ref = oc.hydro_rows(ic["pos"], ic["vel"], full["rho"], full["P"], full["c"], full["h"], ic["m"],
                                      v, 1.0, 2.0, 0.1, rows=rows)
        for k, ref in (("acc_sph", a_ref), ("dudt", du_ref)):
            e = _err(full[k][rows], ref)
            print("lists %s vs oracle: median %.2e max %.2e" % (k, np.median(e), e.max()))
            assert np.median(e) < 1e-5 and e.max() < 1e-3


def test_list_pairs_are_the_support_pairs(oc):
    """With lists every evaluated pair is an in-support pair: the hydro pair
    count equals the oracle's count of j with |r_ij| <= h_i + h_j."""
    from sph_3_b200.ic import evrard
    ic = evrard(6000, seed=12)
    full = _hydro(ic, 128)
    pos, h = ic["pos"], full["h"]
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=2)
    expect = int(np.sum(d <= (h[:, None] + h[None, :])))
    # FP32 cell-relative distances may move pairs that sit exactly on the boundary
    assert abs(full["pairs"] - expect) <= 1e-4 * expect


def test_mixed_pair_sets_vs_exact_fp64_sets(oc):
    """Mixed-precision pair sets (what the hydro pass runs) against the exact
    FP64 support sets {j : |r_ij| <= h_i + h_j} at the same h: the symmetric
    difference is reported; pairs can only differ on the support boundary,
    where the kernel and its gradient vanish."""
    from sph_3_b200 import Config, Context
    from sph_3_b200.ic import evrard
    n = 20000
    ic = evrard(n, seed=13)
    ctx = Context(Config(precision="mixed", gravity=False))
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.compute("boot_h", "h", "density")
    h = ctx.get_field("h")
    rows = np.random.default_rng(2).choice(n, 256, replace=False)
    got = ctx.pair_lists(rows)
    sym = 0
    tot = 0
    for r, g in zip(rows, got):
        ref = oc.neighbours(ic["pos"], h, r)
        sym += np.setxor1d(g, ref).size
        tot += ref.size
        assert np.all(np.diff(g) > 0)
    print("mixed vs exact pair sets: %d of %d pairs differ (%.2e)" % (sym, tot, sym / tot))
    assert sym <= 1e-3 * tot
    ctx.close()


@pytest.mark.parametrize("periodic", [False, True])
def test_fp64_lists_equal_the_walk_bit_for_bit(periodic):
    """The FP64 path's list pass runs the walk's arithmetic in the walk's pair
    order: its hydro results are identical to the walk's."""
    from sph_3_b200 import Config, Context
    if periodic:
        from sph_3_b200.ic import sedov
        ic = sedov(n_side=16, seed=7)
        box, grav = ic["box"], False
    else:
        from sph_3_b200.ic import evrard
        ic = evrard(8000, seed=17)
        box, grav = (0.0, 0.0, 0.0), False
    vel = np.random.default_rng(4).normal(scale=0.3, size=ic["pos"].shape)
    out = []
    for cap in (128, 0):
        ctx = Context(Config(precision="fp64", gravity=grav, box=box, list_cap=cap))
        ctx.set_particles(ic["pos"], ic["m"], vel=vel, u=ic["u"])
        ctx.compute("boot_h", "h", "density")
        ctx.compute("acc_sph", "dudt")
        assert ctx.status() == 0, ctx.status_names()
        out.append((ctx.get_field("acc_sph"), ctx.get_field("dudt"), ctx.get_field("vsig"),
                    ctx.counters()["hydro_pairs"]))
        ctx.close()
    (a1, d1, v1, p1), (a0, d0, v0, p0) = out
    assert np.array_equal(a1, a0) and np.array_equal(d1, d0) and np.array_equal(v1, v0)
    assert p1 < p0  # the list pass runs only the support pairs
