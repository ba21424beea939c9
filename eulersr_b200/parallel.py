"""Case sharding over GPUs (one process per GPU, torch.distributed).

(Mach, alpha) cases are independent, so the solve itself needs no collective:
each rank runs its own batched solver on its shard. The host side here

* splits the case list into per-rank shards balanced by an estimated cost
  (cells x expected iterations; transonic cases, which converge slowest,
  weigh more) with a deterministic longest-processing-time assignment;
* gathers the fixed-size per-case result records to every rank at the end
  (one all_gather over the process group: NCCL between GPUs, gloo on CPU);
* reports a rank that failed: every rank contributes a status word to the
  gather, so the others learn of the failure at the collective instead of
  waiting, and a short process-group timeout bounds the wait if a rank dies;
* averages the warm-start MLP's gradient over ranks for data-parallel
  training (one all_reduce of the flat FP32 gradient per step; every rank
  then takes the same AdamW step, so the replicas stay identical).

This replaces the SLURM job arrays of ``slurm/run_euler_grid.sbatch`` (one
job per angle, a serial Mach loop inside) by one process per GPU.
"""
from __future__ import annotations

import heapq
from dataclasses import dataclass

import numpy as np

RESULT_FIELDS = ("case_index", "status", "converged", "stopping_step", "steps", "n_max", "dt", "last_rel", "cd", "cl",
                 "solve_time_s", "eng_converged", "eng_stopping_step", "final_residual")


def case_cost(mach, n_cells=1.0):
    """Relative cost of a case: cells times an iteration factor that peaks in
    the transonic range (0.8 < M < 1.2)."""
    mach = np.asarray(mach, dtype=np.float64)
    factor = 1.0 + 2.0 * np.exp(-((mach - 1.0) / 0.2) ** 2)
    return np.asarray(n_cells, dtype=np.float64) * factor


def shard_cases(costs, world: int):
    """Deterministic LPT assignment: each case (largest cost first, ties by
    index) goes to the least-loaded rank. Returns a list of index arrays,
    each sorted ascending."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [np.asarray(sorted(s), dtype=np.int64) for s in shards]


def pack_results(results, indices, ok=True):
    """Per-case result dicts -> float64 array (n, len(RESULT_FIELDS)+1); the
    last column carries the rank status word (1 ok, 0 failed)."""
    out = np.zeros((len(indices), len(RESULT_FIELDS) + 1), dtype=np.float64)
    for row, (i, r) in enumerate(zip(indices, results)):
        out[row, 0] = i
        for j, k in enumerate(RESULT_FIELDS[1:], start=1):
            out[row, j] = float(r.get(k, 0.0))
        out[row, -1] = 1.0 if ok else 0.0
    return out


def gather_results(local: np.ndarray, n_total: int, world: int, device="cpu"):
    """All-gather the packed records of every rank; returns (records sorted by
    case index, ranks that reported failure). Ranks pad to the largest shard."""
    import torch
    import torch.distributed as dist
    n_local = torch.tensor([local.shape[0]], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local)
    nmax = int(max(int(s.item()) for s in sizes))
    width = len(RESULT_FIELDS) + 1
    buf = torch.full((max(nmax, 1), width), -1.0, dtype=torch.float64, device=device)
    if local.shape[0]:
        buf[:local.shape[0]] = torch.from_numpy(local).to(device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    rows, failed = [], []
    for r, (p, s) in enumerate(zip(parts, sizes)):
        p = p[: int(s.item())].cpu().numpy()
        if p.shape[0] and np.any(p[:, -1] == 0.0):
            failed.append(r)
        rows.append(p)
    allrows = np.concatenate(rows) if rows else np.zeros((0, width))
    allrows = allrows[np.argsort(allrows[:, 0], kind="stable")]
    return allrows, failed


def records_to_dicts(rows):
    return [{k: (int(v) if k in ("case_index", "status", "converged", "stopping_step", "steps", "n_max",
                                  "eng_converged", "eng_stopping_step") else float(v))
             for k, v in zip(RESULT_FIELDS, row[:-1])} for row in rows]


def allreduce_mean_(t, world: int):
    """In place: the mean of ``t`` over all ranks (sum all_reduce, then / world)."""
    if world <= 1:
        return t
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    t.div_(world)
    return t


def rank_batch(batch: int, world: int, rank: int) -> int:
    """Rows of a global mini-batch that rank ``rank`` draws (equal shares, so
    the mean of the rank means is the global mean)."""
    if batch % world:
        raise ValueError(f"global batch {batch} is not divisible by {world} ranks")
    return batch // world


def solve_sharded(solver_factory, cases, rank: int, world: int, n_cells=1.0, device="cpu"):
    """Solve this rank's shard with ``solver_factory()`` (a Solver) and gather
    every rank's results; returns (all results in case order, failed ranks)."""
    from .solver import FlowCase  # noqa: F401  (cases are FlowCase objects)
    shards = shard_cases(case_cost([c.mach for c in cases], n_cells), world)
    mine = shards[rank]
    ok = True
    results = []
    try:
        if len(mine):
            s = solver_factory()
            results, _ = s.batch_solve([cases[i] for i in mine])
            s.close()
    except Exception:
        ok = False
        results = [{} for _ in mine]
    rows, failed = gather_results(pack_results(results, mine, ok), len(cases), world, device=device)
    return records_to_dicts(rows), failed
