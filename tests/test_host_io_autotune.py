"""Host-side pieces that need no GPU: the reference's raw IC/snapshot layouts,
the seeded IC generators, and the autotuner's candidate grid and cache."""
import json
import os

import numpy as np
import pytest

from sph_3_b200 import autotune, ic, snapio


def _state(n=257, seed=0):
    d = ic.evrard(n, seed=seed)
    d["h"] = np.full(n, 0.05)
    d["eps"] = np.full(n, 0.01)
    d["rho"] = np.linspace(1.0, 2.0, n)
    d["Typ"] = np.zeros(n, dtype=np.int32)
    return d


@pytest.mark.parametrize("writer,reader,size", [(snapio.write_ic, snapio.read_ic, 44),
                                                (snapio.write_ic_header, snapio.read_ic_header, 44),
                                                (snapio.write_snapshot, snapio.read_snapshot, 44)])
def test_round_trip(tmp_path, writer, reader, size):
    st = _state()
    p = str(tmp_path / "f.bin")
    writer(p, st)
    extra = 0 if writer is snapio.write_ic else 4
    assert os.path.getsize(p) == extra + size * st["pos"].shape[0]
    back = reader(p)
    assert np.array_equal(back["pos"], st["pos"].astype(np.float32).astype(np.float64))
    assert np.array_equal(back["m"], st["m"].astype(np.float32).astype(np.float64))
    for k in ("u", "h"):
        assert np.array_equal(back[k], st[k].astype(np.float32).astype(np.float64))


def test_field_order_matches_reference_layouts(tmp_path):
    """Distinct constants per field so a swapped column would show."""
    n = 5
    st = {"pos": np.tile([1.0, 2.0, 3.0], (n, 1)), "vel": np.tile([4.0, 5.0, 6.0], (n, 1)),
          "m": np.full(n, 7.0), "h": np.full(n, 8.0), "eps": np.full(n, 9.0), "u": np.full(n, 10.0),
          "rho": np.full(n, 11.0)}
    p = str(tmp_path / "ic.bin")
    snapio.write_ic(p, st)
    raw = np.fromfile(p, dtype="<f4", offset=4 * n).reshape(10, n)[:, 0]
    assert raw.tolist() == [1, 2, 3, 4, 5, 6, 7, 8, 9, 10]  # x..vz, mass, h, eps, u
    snapio.write_ic_header(p, st)
    raw = np.fromfile(p, dtype="<f4", offset=4 + 4 * n).reshape(10, n)[:, 0]
    assert raw.tolist() == [1, 2, 3, 4, 5, 6, 10, 8, 9, 7]  # x..vz, u, h, eps, mass
    snapio.write_snapshot(p, st)
    raw = np.fromfile(p, dtype="<f4", offset=4 + 4 * n).reshape(10, n)[:, 0]
    assert raw.tolist() == [1, 2, 3, 4, 5, 6, 11, 8, 10, 7]  # x..vz, rho, h, u, mass


def test_non_gas_rejected(tmp_path):
    st = _state(10)
    st["Typ"][3] = 1
    p = str(tmp_path / "s.bin")
    snapio.write_snapshot(p, st)
    with pytest.raises(ValueError):
        snapio.read_snapshot(p)
    assert snapio.read_snapshot(p, allow_non_gas=True)["Typ"][3] == 1


def test_ic_generators_shapes_and_seeds():
    a, b = ic.evrard(1000, seed=3), ic.evrard(1000, seed=3)
    assert np.array_equal(a["pos"], b["pos"])
    r = np.linalg.norm(a["pos"], axis=1)
    assert r.max() <= 1.0 and abs(a["m"].sum() - 1.0) < 1e-12
    s = ic.sedov(n_side=8, seed=1)
    assert s["pos"].shape == (512, 3) and s["pos"].min() >= 0 and s["pos"].max() < 1.0
    e_dep = np.sum(s["m"] * (s["u"] - 1e-5))
    assert abs(e_dep - 1.0) < 1e-9
    k = ic.kelvin_helmholtz(n=5000, seed=0)
    assert k["pos"].shape == (5000, 3) and k["pos"][:, 2].max() < 1.0 / 16.0
    bt = ic.evrard_batch(ncloud=16, seed=2, n_min=100, n_max=1000)
    assert bt["pos"].shape[0] == bt["counts"].sum() and len(bt["counts"]) == 16
    assert np.all((bt["counts"] >= 100) & (bt["counts"] <= 1000))


def test_autotune_grid_respects_stack_bound():
    cands = list(autotune.candidates({"stack_cap": (64, 256, 512), "leaf_size": (8, 16)}, max_level=16))
    assert all(c["stack_cap"] >= 7 * 18 + 32 for c in cands)
    assert len(cands) == 4


def test_autotune_cache_roundtrip(tmp_path, monkeypatch):
    monkeypatch.setenv("SPH3_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    key = autotune.workload_key("NVIDIA B200", 1048576, 1, "mixed", False)
    assert key == "NVIDIA B200|n2^20|clouds2^0|mixed|open"
    autotune.save_cache({key: {"best": {"leaf_size": 16}, "ms_per_step": 11.0}})
    assert autotune.load_cache()[key]["best"]["leaf_size"] == 16
    json.loads(open(str(tmp_path / "cache.json")).read())
