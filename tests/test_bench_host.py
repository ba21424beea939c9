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


def test_warm_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    made = _fake_meshes(monkeypatch)
    args = types.SimpleNamespace(workload="warm", steps=3, warmup=3)
    assert bench.run_reference_warm(args, 2, 1) == 0
    assert made == [] and capsys.readouterr().out == ""


def test_warm_cases_are_the_held_out_draws_sharded_by_cost():
    """The held-out cases follow the training draws of default_rng(3); under
    two ranks the product's cost-balanced scheduler deals 2 x n_eval draws
    without overlap and with balanced estimated cost."""
    from eulersr_b200.parallel import case_cost
    from eulersr_b200.warmstart.pipeline import draw_cases
    args = types.SimpleNamespace(n_train=16, n_eval=8)
    idx, me, ae = bench.warm_cases(args, 1, 0)
    _, (me1, ae1) = draw_cases(16, 8, seed=3)
    assert list(idx) == list(range(8)) and np.array_equal(me, me1) and np.array_equal(ae, ae1)
    i0, m0, _ = bench.warm_cases(args, 2, 0)
    i1, m1, _ = bench.warm_cases(args, 2, 1)
    assert len(i0) + len(i1) == 16 and not (set(i0) & set(i1))
    c0, c1 = case_cost(m0).sum(), case_cost(m1).sum()
    assert abs(c0 - c1) <= case_cost(np.r_[m0, m1]).max()


def test_cpu_converged_sample_rule(diamond02):
    """The host arm's stop rule: a case stops once its CD stayed within the
    tolerance of its reference for `patience` checks; an unreachable
    reference runs to the cap and does not count."""
    from oracle import euler_oracle as O
    from oracle.cport import CpuCase
    cc = CpuCase(diamond02, 2.5, 5.0, np.float32)
    W = cc.srk2_local(cc.W0, 100, 0.6)
    cd100 = float(O.force_coefficients(W.astype(np.float64), cc.om, 1.0, 2.5 * 1.4 ** 0.5,
                                       diamond02.metadata.get("obstacle_length", 1.0))[0])
    n, t, recs, thr = bench.cpu_converged_sample(
        [{"mach": 2.5, "aoa": 5.0, "cd": cd100 * 10, "steady": True}], 1e9, diamond02, patience=2, max_steps=100)
    assert n == 0 and recs[0]["steps"] == 100 and not recs[0]["converged"]
    n, t, recs, thr = bench.cpu_converged_sample(
        [{"mach": 2.5, "aoa": 5.0, "cd": cd100, "steady": True}], 1e9, diamond02, cd_tol=0.2, patience=2,
        max_steps=400)
    assert recs[0]["steps"] <= 400 and thr >= 1


def _shard_rank_main(rank, world, port, q):
    import os
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from eulersr_b200.parallel import case_cost
        args = types.SimpleNamespace(n_train=32, n_eval=16)
        idx, me, ae = bench.warm_cases(args, world, rank)
        n = bench.allreduce_sum(float(len(idx)), world)
        cmax = bench.allreduce_max(float(case_cost(me).sum()), world)
        csum = bench.allreduce_sum(float(case_cost(me).sum()), world)
        got = [None] * world
        dist.all_gather_object(got, sorted(int(i) for i in idx))
        q.put((rank, n, cmax, csum, got))
    finally:
        dist.destroy_process_group()


def test_warm_shards_over_two_gloo_ranks():
    """Under two ranks (gloo here, NCCL on GPUs) the held-out draws are dealt
    by the cost-balanced scheduler: every draw to exactly one rank, the
    slowest rank's estimated cost within one case of the mean."""
    import multiprocessing as mp
    import socket
    from eulersr_b200.parallel import case_cost
    from eulersr_b200.warmstart.pipeline import draw_cases
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_shard_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, n, cmax, csum, got), _ = out
    assert n == 32
    assert sorted(got[0] + got[1]) == list(range(32))
    _, (me, _) = draw_cases(32, 32, seed=3)
    assert cmax - csum / 2 <= case_cost(me).max()


def test_plain_truth_table_covers_throughput_cases():
    """The committed float64 references of the throughput workload's NACA0012 cases (the
    bench's converged-cases leg reads them) cover exactly the 256 cases the
    throughput workload draws, with finite CDs and a steady flag each
    (subsonic inviscid cases have near-zero drag, a few slightly negative
    from the discretisation)."""
    import json
    import bench
    rows = json.loads(bench.PLAIN_TRUTH_FILE.read_text())["cases"]
    mach, aoa = bench.batch_cases(256)
    want = {(round(float(m), 12), round(float(a), 12)) for m, a in zip(mach, aoa)}
    got = {(round(r["mach"], 12), round(r["aoa"], 12)) for r in rows}
    assert got == want
    assert all(np.isfinite(r["cd"]) and abs(r["cd"]) < 1.0 and isinstance(r["steady"], bool) for r in rows)


class _FakeWF:
    """Stands in for the GPU warm-start workflow: fixed step counts per start,
    every fifth case capped, every seventh a fallback."""

    def __init__(self, **kw):
        self.cd_tol, self.schedule, self.unsteady_cap, self.warm_budget = 0.005, "fifo", None, 3000
        self.hr = types.SimpleNamespace(n_cells=100)
        self.lr = types.SimpleNamespace(n_cells=20)
        self.calls = []

    def prepare(self, **kw):
        return {"n_train": kw.get("n_train")}

    def truth(self, me, ae):
        return np.full(len(me), 0.05), np.arange(len(me)) % 4 != 0

    def solve(self, me, ae, truth, steady, start="mlp", want_states=False):
        from eulersr_b200.warmstart import workflow as W
        self.calls.append(start)
        n = len(me)
        steps = {"mlp": 900, "idw": 1200, "cold": 2800, "single": 2800}[start]
        res = [{"status": 2 if i % 5 else 3, "cd": float(truth[i]), "cl": 0.0, "steps": steps,
                "stopping_step": steps, **({"fallback": True, "warm_steps": 3000} if i % 7 == 0 else {})}
               for i in range(n)]
        conv = sum(1 for i in range(n) if res[i]["status"] == 2 and steady[i])
        sec = {"mlp": 1.0, "idw": 1.2, "cold": 1.5, "single": 10.0}[start]
        return W.PassResult(start, res, conv, sec, sec, {"hr_solve_s": sec}, [steps] * n,
                            [np.zeros((100, 4))] * n if want_states else None)

    def solve_stream(self, batches, truth_of, steady_of, use_mlp=True):
        out = [self.solve(m, a, t, s) for (m, a), t, s in zip(batches, truth_of, steady_of)]
        return out, 0.9 * len(out), 0.9 * len(out)

    def kernel_launches(self):
        return 10 * len(self.calls)

    def close(self):
        pass


class _FakeClock:
    def __init__(self, *a):
        pass

    def start(self):
        pass

    def stop(self):
        return {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}


def _install_warm_fakes(put):
    """The headline path's GPU pieces replaced by fakes (put = setattr, or
    pytest's monkeypatch.setattr)."""
    import torch
    from eulersr_b200.warmstart import workflow as W
    thr = {"value": 1e10, "unit": "cell-updates/s", "ms_per_step": 25.0, "alg_gbs_per_step": 1.0,
           "alg_bytes_per_cell_update": 80.5, "e2e": {"value": 9e9}, "kernel_times_ms": {}, "config": {},
           "roofline": {"frac": 0.28}, "gpu_launches": 400}
    put(W, "WarmStartWorkflow", _FakeWF)
    put(bench, "ClockSampler", _FakeClock)
    put(bench, "run_throughput", lambda *a, **k: dict(thr))
    put(bench, "run_plain_converged", lambda *a, **k: {"value": 50.0})
    put(torch.cuda, "set_device", lambda *a: None)
    put(torch.cuda, "synchronize", lambda *a: None)
    put(torch.cuda, "empty_cache", lambda *a: None)
    real_empty = torch.empty
    put(torch, "empty", lambda *a, **k: real_empty(8, dtype=k.get("dtype")))


def _warm_args():
    return types.SimpleNamespace(slots=32, max_steps=12000, lr_steps=2000, warm_budget=3000, make_truth=False,
                                 n_train=16, n_eval=12, target_steps=100, train_steps=10, steps=2, warmup=3,
                                 unsteady_cap=3000, no_cpu=True, workload="warm", cases=256, chunk=50, h=0.025,
                                 block=0, no_e2e=False, precision="f32", make_plain_truth=False)


def test_warm_headline_line_on_fakes(monkeypatch, capsys):
    """The headline workload end to end on CPU with a fake workflow in place
    of the GPU one: every leg runs, and the JSON line carries the contract's
    keys, the ratios and the per-case / by-class breakdowns."""
    import json
    _install_warm_fakes(monkeypatch.setattr)
    assert bench.run_warm(_warm_args(), 1, 0, 0) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "cpu_baseline", "clocks",
                "gpu_launches"):
        assert key in line, key
    c = line["converged_cases_per_s"]
    assert c["ratio_warm_vs_plain_single_case"] == line["value"] / c["plain_single_case"]
    assert len(c["per_case"]["mlp"]["steps"]) == 12 and set(c["per_case"]) >= {"single", "cold", "idw", "mlp"}
    assert sum(b["cases"] for b in c["by_case_class"]["by_mach_band"]) == 12
    assert c["plain_batched_naca0012_x256"] == {"value": 50.0}
    assert c["warm_mlp_streamed"]["batches"] == 2 and c["unsteady_capped_protocol"]["unsteady_cap_steps"] == 3000


def _warm_rank_main(rank, world, port, q):
    import contextlib
    import datetime
    import io
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        _install_warm_fakes(setattr)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            rc = bench.run_warm(_warm_args(), world, rank, 0)
        q.put((rank, rc, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_warm_headline_over_two_gloo_ranks():
    """The headline path under two ranks (gloo here, NCCL on GPUs), on the
    fake workflow: both ranks take the same collective steps and finish, rank
    0 alone prints the line, whose value is the converged cases of both ranks
    over the slower rank's time."""
    import json
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_warm_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, rc0, text0), (r1, rc1, text1) = out
    assert (rc0, rc1) == (0, 0) and text1.strip() == ""
    line = json.loads(text0.strip().splitlines()[-1])
    assert line["n_gpus"] == 2
    passes = line["converged_cases_per_s"]["warm_passes"]
    assert line["value"] > 0 and len(passes) == 2


class _FakeSolver:
    """Stands in for the GPU solver in the throughput workload: each chunk
    'takes' 25 ms; transfers and tuning are no-ops."""

    def __init__(self, meshes, slots, **kw):
        self.n = int(slots) if np.isscalar(slots) else int(sum(slots))
        self.cells = 1000

    def set_cases(self, slots, cases, fields=None):
        pass

    def synchronize(self):
        pass

    def tuning(self):
        return {"block_size": 128, "k2_patches": True, "step_ms": {}, "variants": []}

    def step(self, n):
        self.last = n

    def elapsed_ms(self):
        return 25.0

    def kernel_launches(self):
        return 0

    def profile_step(self, n=8):
        return {"recon_ms": 0.11, "flux_ms": 0.14, "other_ms": 0.0, "recon_launches": 1, "flux_launches": 1,
                "other_launches": 0}

    def _n_cells(self, b):
        return self.cells

    def stage_cases(self, slots, cases, fields):
        pass

    def apply_staged(self):
        pass

    def fetch_states(self, slots, out):
        return out

    def wait_transfers(self):
        pass

    def close(self):
        pass


def _throughput_rank_main(rank, world, port, q):
    import contextlib
    import datetime
    import io
    import os
    import torch.distributed as dist
    from eulersr_b200 import solver as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        setattr(S, "Solver", _FakeSolver)
        setattr(S, "DeviceMesh", lambda m: m)
        setattr(bench, "ClockSampler", _FakeClock)
        setattr(bench, "get_mesh", lambda geom, h: types.SimpleNamespace(n_cells=1000, geom=geom, h=h))
        args = types.SimpleNamespace(workload="naca", cases=64, chunk=50, h=0.025, steps=2, warmup=3, block=0,
                                     no_e2e=False, no_cpu=True, gpus=world)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            out = bench.run_throughput(args, world, rank, 0, report=True)
        q.put((rank, out["value"], out["config"]["cases_this_rank"], buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_throughput_over_two_gloo_ranks():
    """The throughput workload under two ranks on a fake solver: each rank
    takes its share of the cases by the cost-balanced scheduler, the value is
    every rank's cell-updates over the slower rank's time, and rank 0 alone
    prints the line."""
    import json
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_throughput_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, v0, n0, text0), (r1, v1, n1, text1) = out
    assert n0 + n1 == 128 and v0 == v1
    assert v0 == 1000 * 128 * 50 * 2 / (2 * 25.0 * 1e-3)
    assert text1.strip() == "" and json.loads(text0.strip().splitlines()[-1])["n_gpus"] == 2
