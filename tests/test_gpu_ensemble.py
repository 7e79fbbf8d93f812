"""The batched-ensemble configuration as specified: 256 independent Evrard
clouds with N log-uniform in [2,048, 65,536] (seeded, about 5M particles),
each with its own M and R in [0.5, 2], stepped together by one launch
sequence per pass under a CUDA-graph-captured step, with the walk launch
parameters chosen by the autotuner, FP32 mixed precision.  Eight clouds
spanning the size range are checked against per-cloud runs of the plain
FP64 GPU path (same theta = 0.5): positions after two steps within 1e-6 of
the cloud's radius, densities within 1e-3 (median; the two h searches settle
differently inside the same window), and the ensemble's mass conserved."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_256_cloud_ensemble_autotuned_vs_per_cloud_fp64(tmp_path, monkeypatch):
    monkeypatch.setenv("SPH3_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    from sph_3_b200 import Config, Context, autotune
    from sph_3_b200.ic import evrard_batch
    b = evrard_batch(ncloud=256, seed=0, n_min=2048, n_max=65536)
    counts = b["counts"]
    assert counts.min() >= 2048 and counts.max() <= 65536 and 4e6 < counts.sum() < 7e6
    ctx = Context(Config(precision="mixed", use_graph=True))
    ctx.set_clouds(counts)
    ctx.set_particles(b["pos"], b["m"], vel=b["vel"], u=b["u"])
    ctx.first_step(1e-3)
    best, times = autotune.autotune(ctx, steps=2, warmup=2,
                                    grid={"leaf_size": (12, 16, 24), "walk_warps": (2, 4), "stack_cap": (768,)})
    assert len(times) == 6 and ctx.config.leaf_size == best["leaf_size"]
    print("ensemble autotune: best %s, ms/step %s" % (best, {k: round(v, 2) for k, v in times.items()}))
    ctx.step(1e-3, 2)
    assert ctx.status() == 0, ctx.status_names()
    assert ctx.kernels_per_step() > 0  # the step ran as a captured graph
    pos, rho = ctx.get_field("pos"), ctx.get_field("rho")
    e = ctx.energy()
    assert abs(e["M"] - b["M"].sum()) < 1e-9 * b["M"].sum()
    ctx.close()
    begin = np.concatenate([[0], np.cumsum(counts)[:-1]])
    picks = np.argsort(counts)[np.linspace(0, counts.size - 1, 8).astype(int)]
    for k in picks:
        sl = slice(int(begin[k]), int(begin[k] + counts[k]))
        one = Context(Config(precision="fp64", use_graph=False))
        one.set_particles(b["pos"][sl], b["m"][sl], vel=b["vel"][sl], u=b["u"][sl])
        one.first_step(1e-3)
        one.step(1e-3, 2)
        assert one.status() == 0
        dpos = np.abs(pos[sl] - one.get_field("pos")).max() / b["R"][k]
        drho = np.median(np.abs(rho[sl] / one.get_field("rho") - 1.0))
        print("cloud %d (N=%d): max |dpos|/R %.2e, median |drho/rho| %.2e" % (k, counts[k], dpos, drho))
        assert dpos < 1e-6
        assert drho < 1e-3
        one.close()
