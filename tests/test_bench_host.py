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


def _rank_main(rank, world, port, q):
    import os
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        t = bench.allreduce_max(1.5 + rank, world)
        s = bench.allreduce_sum(10.0 * (rank + 1), world)
        q.put((rank, t, s))
    finally:
        dist.destroy_process_group()


def test_bench_reductions_over_two_ranks():
    """The job time is the max over ranks and the work the sum, as bench.py
    reduces them under torchrun (gloo here, NCCL on GPUs)."""
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2.5, 30.0), (1, 2.5, 30.0)]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun the reference arm's other ranks exit 0 at once: no mesh,
    no CPU work, no JSON line."""
    made = _fake_meshes(monkeypatch)
    args = types.SimpleNamespace(workload="naca", h=0.025, cases=256, steps=3, warmup=3, precision="f32")
    assert bench.run_reference(args, 2, 1) == 0
    assert made == [] and capsys.readouterr().out == ""
