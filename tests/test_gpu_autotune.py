"""Autotuner on the GPU: times a small grid on the caller's particles,
applies the best candidate and leaves the particle state as it found it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_applies_best_and_restores_state(tmp_path, monkeypatch):
    monkeypatch.setenv("SPH3_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    from sph_3_b200 import Config, Context, autotune
    from sph_3_b200.ic import evrard
    ic = evrard(30000, seed=6)
    ctx = Context(Config())
    ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
    ctx.first_step(1e-3)
    before = ctx.get_field("pos")
    best, times = autotune.autotune(ctx, steps=2, warmup=2,
                                    grid={"leaf_size": (8, 16), "walk_warps": (2, 4), "stack_cap": (512,)})
    assert len(times) == 4 and best in [dict(leaf_size=l, walk_warps=w, stack_cap=512)
                                        for l in (8, 16) for w in (2, 4)]
    assert ctx.config.leaf_size == best["leaf_size"] and ctx.config.walk_warps == best["walk_warps"]
    assert np.array_equal(ctx.get_field("pos"), before)
    # a second call is served from the cache
    best2, _ = autotune.autotune(ctx, steps=2, warmup=2)
    assert best2 == best
    ctx.step(1e-3, 2)
    assert ctx.status() == 0
    ctx.close()


@pytest.mark.parametrize("warps", [1, 2, 8])
def test_walk_width_does_not_change_results(warps):
    from sph_3_b200 import Config, Context
    from sph_3_b200.ic import evrard
    ic = evrard(20000, seed=8)
    out = []
    for w in (4, warps):
        ctx = Context(Config(precision="fp64", walk_warps=w))
        ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
        ctx.first_step(1e-3)
        out.append((ctx.get_field("rho"), ctx.get_field("acc")))
        ctx.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
