"""Host logic of bench.py on CPU: the ragged multi-mesh workload (12 meshes,
1024 cases dealt round-robin, seeded draws), the single-case diamond
settings and the config block of the JSON line."""
import types

import numpy as np

import bench


def _fake_meshes(monkeypatch):
    made = []

    def get_mesh(geom, h):
        m = types.SimpleNamespace(n_cells=int(1000 / h), geom=geom, h=h)
        made.append((geom, h))
        return m
    monkeypatch.setattr(bench, "get_mesh", get_mesh)
    return made


def test_ragged_workload_deals_1024_cases_round_robin(monkeypatch):
    made = _fake_meshes(monkeypatch)
    meshes, per = bench.ragged_workload()
    assert len(meshes) == 12 and len(set(made)) == 12
    assert sum(len(p) for p in per) == 1024
    assert [len(p) for p in per] == [86] * 4 + [85] * 8
    rng = np.random.default_rng(2)
    mach, aoa = rng.uniform(0.7, 3.0, 1024), rng.uniform(-5.0, 5.0, 1024)
    assert per[0][0] == (float(mach[0]), float(aoa[0])) and per[1][0] == (float(mach[1]), float(aoa[1]))
    assert per[0][1] == (float(mach[12]), float(aoa[12]))
    # two ranks split the 2048 draws between them without overlap
    _, r0 = bench.ragged_workload(rank=0, world=2)
    _, r1 = bench.ragged_workload(rank=1, world=2)
    a = {c for p in r0 for c in p}
    b = {c for p in r1 for c in p}
    assert len(a) == len(b) == 1024 and not (a & b)


def test_config_blocks(monkeypatch):
    _fake_meshes(monkeypatch)
    args = types.SimpleNamespace(workload="ragged", chunk=50, h=0.025, cases=256)
    meshes, per = bench.ragged_workload()
    cfg = bench.workload_config(args, (meshes, per))
    assert cfg["cases_per_gpu"] == 1024 and len(cfg["cells"]) == 12 and "ragged" in cfg["workload"]
    args.workload = "naca"
    cfg = bench.workload_config(args, types.SimpleNamespace(n_cells=25049))
    assert cfg["cells"] == 25049 and cfg["cases_per_gpu"] == 256


def test_diamond_single_case_settings():
    assert bench.diamond_case(0.1)[:4] == (2.5, 5.0, 0.8, "density_l2")
    assert bench.diamond_case(0.025)[:4] == (2.0, 0.0, 0.6, "reference")
