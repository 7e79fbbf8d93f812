"""sph3_step_io: one KDK step with the reference loop's state (r, v, acc, h,
u, ut_previous) in host memory, moved in and out in the same call with the
transfers overlapping the step.  It must give, bit for bit, what the
field-by-field path gives (sph3_set_field x6 -> sph3_step -> sph3_get_field
x6) on a context with the same history, for both precisions and step
orders, with page-locked and pageable host buffers, and at a size where the
first inputs and the closing outputs move in row chunks (ragged last chunk)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "acc", "h", "u", "dudt_prev")
OUTS = ("pos", "vel", "acc", "h", "u", "dudt_prev", "rho", "nngb")


def _ctx(cfg, ic):
    from sph_3_b200 import Context
    ctx = Context(cfg)
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.first_step(1e-3)
    ctx.step(1e-3, 1)
    return ctx


@pytest.mark.parametrize("prec,order,pinned,n", [("mixed", "serial", True, 30000), ("fp64", "serial", False, 30000),
                                                 ("mixed", "mpi4", True, 30000), ("mixed", "serial", True, 70001),
                                                 ("fp64", "serial", True, 70001), ("mixed", "mpi4", False, 70001)])
def test_step_io_matches_field_by_field(prec, order, pinned, n):
    import torch
    from sph_3_b200 import Config
    from sph_3_b200.ic import evrard
    ic = evrard(n, seed=13)
    ic["vel"] = np.random.default_rng(13).normal(scale=0.05, size=(n, 3))
    cfg = Config(precision=prec, step_order=order, visc="balsara" if order == "mpi4" else "signal")
    a, b = _ctx(cfg, ic), _ctx(cfg, ic)
    state = {f: a.get_field(f) for f in FIELDS}
    # field by field
    for f in FIELDS:
        a.set_field(f, state[f])
    a.step(1e-3, 1)
    want = {f: a.get_field(f) for f in OUTS}
    # one call, host buffers
    if pinned:
        ins = {f: torch.from_numpy(state[f]).pin_memory() for f in FIELDS}
        outs = {f: torch.empty(want[f].shape, dtype=torch.float64).pin_memory() for f in OUTS}
    else:
        ins = dict(state)
        outs = {f: np.empty_like(want[f]) for f in OUTS}
    b.step_io(1e-3, ins, outs)
    for f in OUTS:
        got = outs[f].numpy() if hasattr(outs[f], "numpy") else outs[f]
        assert np.array_equal(got, want[f]), f
    assert a.status() == 0 and b.status() == 0
    # a second call with the same buffers (page-locked: a replayed graph) and
    # the next state written into them
    state2 = {f: a.get_field(f) for f in FIELDS}
    for f in FIELDS:
        a.set_field(f, state2[f])
    a.step(1e-3, 1)
    want2 = {f: a.get_field(f) for f in OUTS}
    for f in FIELDS:
        if hasattr(ins[f], "numpy"):
            ins[f].numpy()[...] = state2[f]
        else:
            ins[f][...] = state2[f]
    b.step_io(1e-3, ins, outs)
    for f in OUTS:
        got = outs[f].numpy() if hasattr(outs[f], "numpy") else outs[f]
        assert np.array_equal(got, want2[f]), f
    # the context goes on from the state the call left (graph steps after an I/O step)
    a.step(1e-3, 2)
    b.step(1e-3, 2)
    assert np.array_equal(a.get_field("pos"), b.get_field("pos"))
    a.close()
    b.close()


def test_step_io_rejects_bad_fields():
    from sph_3_b200 import Config
    from sph_3_b200._lib import Sph3Error
    from sph_3_b200.ic import evrard
    ic = evrard(2000, seed=1)
    ctx = _ctx(Config(), ic)
    with pytest.raises(ValueError):
        ctx.step_io(1e-3, {"pos": np.zeros((10, 3))}, {})
    import ctypes
    fi = (ctypes.c_int32 * 1)(99)
    buf = np.zeros(6000)
    pi = (ctypes.c_void_p * 1)(buf.ctypes.data)
    rc = ctx.lib.sph3_step_io(ctx._ptr, 1e-3, 1, 1, fi, pi, 0, None, None, None)
    assert rc == 1  # SPH3_ERR_INVALID_ARG
    with pytest.raises(Sph3Error):
        from sph_3_b200._lib import check
        check(ctx.lib.sph3_step_io(ctx._ptr, 1e-3, 0, 0, None, None, 0, None, None, None))
    ctx.close()
