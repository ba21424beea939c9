"""Multi-rank case sharding on CPU (gloo, world size 2): shard balance, the
all-gather of result records, and failure reporting when a rank's solve
raises or a rank never joins the collective. No GPU involved."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from eulersr_b200.parallel import (RESULT_FIELDS, case_cost, gather_results, pack_results, records_to_dicts,
                                   shard_cases)


def test_shards_cover_every_case_once_and_balance():
    rng = np.random.default_rng(1)
    mach = rng.uniform(0.7, 3.0, 257)
    costs = case_cost(mach, 25000)
    for world in (1, 2, 3, 8):
        shards = shard_cases(costs, world)
        allidx = np.sort(np.concatenate(shards))
        assert np.array_equal(allidx, np.arange(257))
        loads = [costs[s].sum() for s in shards]
        assert max(loads) - min(loads) <= costs.max() + 1e-9
    assert [s.tolist() for s in shard_cases(costs, 4)] == [s.tolist() for s in shard_cases(costs, 4)]


def test_transonic_costs_more():
    c = case_cost([0.7, 1.0, 2.5])
    assert c[1] > c[0] > c[2] * 0.99


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        n = 11
        shards = shard_cases(case_cost(np.linspace(0.7, 3.0, n)), world)
        mine = shards[rank]
        ok = not (mode == "raise" and rank == 1)
        res = [{"status": 2, "converged": 1, "stopping_step": int(100 + i), "steps": int(100 + i), "n_max": 1000,
                "dt": 1e-3, "last_rel": 1e-7, "cd": 0.01 * i, "cl": 0.0, "solve_time_s": 0.1} for i in mine]
        if mode == "hang" and rank == 1:
            # this rank never reaches the collective (it exits between steps)
            q.put((rank, "left", None))
            return
        rows, failed = gather_results(pack_results(res, mine, ok), n, world)
        q.put((rank, "ok", (records_to_dicts(rows), failed)))
    except Exception as e:  # the collective ended with an error (timeout / peer gone)
        q.put((rank, "error", type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(2):
        r, kind, val = q.get(timeout=120)
        out[r] = (kind, val)
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_gather_results_two_ranks():
    out = _run("ok")
    for r in (0, 1):
        kind, (rows, failed) = out[r]
        assert kind == "ok" and failed == []
        assert [d["case_index"] for d in rows] == list(range(11))
        assert [d["stopping_step"] for d in rows] == [100 + i for i in range(11)]
        assert set(rows[0]) == set(RESULT_FIELDS)


def test_failed_rank_is_reported():
    out = _run("raise")
    for r in (0, 1):
        kind, (rows, failed) = out[r]
        assert kind == "ok" and failed == [1]


def test_rank_that_leaves_ends_the_collective_with_an_error():
    out = _run("hang")
    assert out[1][0] == "left"
    assert out[0][0] == "error"


def _dp_worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    from eulersr_b200.parallel import allreduce_mean_, rank_batch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        g = torch.arange(6, dtype=torch.float32) * (rank + 1)      # this rank's gradient
        allreduce_mean_(g, world)
        q.put((rank, g.tolist(), rank_batch(32768, world, rank)))
    finally:
        dist.destroy_process_group()


def test_data_parallel_gradient_mean():
    """Gradient averaging of data-parallel MLP training over two gloo ranks:
    both ranks end with the same mean, so their AdamW steps stay identical."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_dp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict((r, (g, b)) for r, g, b in (q.get(timeout=120) for _ in range(2)))
    for p in ps:
        p.join(timeout=60)
    expect = [1.5 * i for i in range(6)]
    assert got[0][0] == expect and got[1][0] == expect
    assert got[0][1] == got[1][1] == 16384
    import pytest
    from eulersr_b200.parallel import rank_batch
    with pytest.raises(ValueError):
        rank_batch(100, 3, 0)
