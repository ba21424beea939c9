"""The warm-start workflow as one reusable object (evaluation and bench).

Converged HR cases per second at a CD accuracy, for four ways of reaching a
converged HR field of each (Mach, alpha) case:

* ``mlp``    LR solve of every case -> LR pressure gradients -> IDW (k=6, p=2)
             + residual MLP on the GPU -> HR solve from that prediction
             (eval/convergence_case.py:106-140: the whole pipeline is timed);
             a case the rule has not stopped within ``warm_budget`` steps
             restarts from freestream with the rest of the step cap;
* ``idw``    the same without the MLP;
* ``cold``   HR solve from freestream, ``slots`` cases at a time with
             retire/refill;
* ``single`` HR solve from freestream one case at a time (one slot), the
             plain single-case solve.

Every HR solve runs the local CFL step and ends a case once its CD has stayed
within ``cd_tol`` of that case's reference CD for ``patience`` checks
``check_every`` steps apart, or at ``max_steps``. A case counts as converged
when the rule stopped it, its reference is steady and the CD it stopped at is
within ``cd_tol`` of the reference. The reference CD of a case comes from a
long float64 solve of the same kernels (``truth``): ``ref_steps`` steps, then
``confirm_steps`` more; a reference whose CD still moves by more than 0.1 %
marks the case unsteady (a failure for every start).

Solvers are created once and reused, so a timed pass contains no solver
set-up, autotuning or mesh upload.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from ..meshing.generate import cached_mesh
from ..solver import DeviceMesh, FlowCase, Solver
from .features import MeshPair
from .mlp import MLP
from .pipeline import WarmStart, build_training_set, draw_cases, eval_loss, pressure_gradients, primitives, train


@dataclass
class PassResult:
    start: str
    results: list
    converged: int
    seconds: float                 # device timeline of the pass (CUDA events, device synchronised)
    wall_s: float
    parts_s: dict = field(default_factory=dict)
    iterations: list = field(default_factory=list)
    states: list | None = None

    @property
    def cases_per_s(self) -> float:
        return self.converged / self.seconds if self.seconds > 0 else 0.0


def _device_timed(fn):
    """Run fn() between two CUDA events recorded after a device-wide
    synchronisation (the events bracket every stream's work); returns
    (fn(), device seconds, wall seconds)."""
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    e1.record()
    e1.synchronize()
    return out, e0.elapsed_time(e1) * 1e-3, time.perf_counter() - t0


class WarmStartWorkflow:
    def __init__(self, geom="naca2412", h_hr=0.025, h_lr=0.1, slots=32, lr_steps=2000, max_steps=12000,
                 check_every=25, patience=8, cd_tol=0.005, device=0, schedule="fifo",
                 warm_budget=3000, unsteady_cap=None):
        self.hr, self.lr = cached_mesh(geom, h_hr), cached_mesh(geom, h_lr)
        self.pair = MeshPair.build(self.hr, self.lr)
        self.dm_hr, self.dm_lr = DeviceMesh(self.hr), DeviceMesh(self.lr)
        self.slots, self.lr_steps, self.max_steps = slots, lr_steps, max_steps
        self.check_every, self.patience, self.cd_tol = check_every, patience, cd_tol
        self.device = device
        if schedule not in ("lr_longest_first", "fifo"):
            raise ValueError("schedule must be 'lr_longest_first' or 'fifo'")
        self.schedule = schedule
        self.warm_budget = warm_budget   # None or 0: no fallback to freestream
        self.unsteady_cap = unsteady_cap   # None: unsteady-flagged cases run to max_steps too
        self.ws = WarmStart(self.pair, device=f"cuda:{device}")
        self._solvers = {}
        self.train_info = {}

    # --------------------------------------------------------------- solvers
    def _solver(self, key, dm, slots, **kw):
        s = self._solvers.get(key)
        if s is None:
            s = Solver(dm, slots, device=self.device, **kw)
            self._solvers[key] = s
        return s

    def _hr_solver(self, slots):
        return self._solver(("hr", slots), self.dm_hr, slots, precision="f32", dt_mode="local",
                            stop_rule="engineering", threshold=1e-30, check_every=self.check_every,
                            patience=self.patience)

    # the LR side runs at the device's highest stream priority: in a stream of
    # batches its short launches get SMs ahead of the HR batch's chunks
    def _lr_solver(self, slots):
        return self._solver(("lr", slots), self.dm_lr, slots, precision="f32", dt_mode="local", stop_rule="reference",
                            threshold=1e-30, check_every=self.check_every, patience=self.patience,
                            stream_priority=-100)

    def _grad_solver(self):
        return self._solver(("grad",), self.dm_lr, 1, precision="f64", stream_priority=-100)

    def _cases(self, machs, aoas, targets=None, max_steps=None, dtype=np.float32):
        """FlowCases; max_steps: None (the workflow's cap), one cap, or one per case."""
        caps = np.broadcast_to(np.asarray(self.max_steps if max_steps is None else max_steps, dtype=np.int64),
                               (len(machs),))
        out = []
        for i, (m, a) in enumerate(zip(machs, aoas)):
            kw = {}
            if targets is not None:
                kw = dict(eng_target_cd=float(targets[i]), eng_target_cl=0.0, eng_cd_tol=self.cd_tol,
                          eng_cl_tol=1e12, eng_patience=self.patience)
            out.append(FlowCase(mach=float(m), aoa_deg=float(a), cfl=0.6, tf=1e9,
                                max_steps=int(caps[i]), dtype=dtype, **kw))
        return out

    def caps(self, steady):
        """Step cap of each HR case: ``max_steps``, or ``unsteady_cap`` for a
        case whose reference is flagged unsteady (it counts as a failure for
        every start whatever it does, so every start stops it there)."""
        steady = np.asarray(steady, dtype=bool)
        c = np.full(len(steady), self.max_steps, dtype=np.int64)
        if self.unsteady_cap:
            c[~steady] = min(self.max_steps, int(self.unsteady_cap))
        return c

    def close(self):
        for s in self._solvers.values():
            s.close()
        self._solvers.clear()

    def kernel_launches(self) -> int:
        """Library kernels launched so far by this workflow's solvers and its
        IDW, feature, MLP and decode calls."""
        return sum(s.kernel_launches() for s in self._solvers.values()) + self.ws.launches + (
            self.ws.mlp.launches if self.ws.mlp is not None else 0)

    # ----------------------------------------------------------------- set-up
    def lr_solutions(self, machs, aoas, with_results=False):
        """LR fields of every case (fixed lr_steps) and their LSQ pressure
        gradients (and the LR solve's per-case results)."""
        s = self._lr_solver(len(machs))
        res, states = s.batch_solve(self._cases(machs, aoas, max_steps=self.lr_steps), want_states=True)
        g = self._grad_solver()
        grads = []
        for W, m, a in zip(states, machs, aoas):
            g.set_case(0, FlowCase(mach=float(m), aoa_deg=float(a), tf=1.0), W_init=W)
            grads.append(g.gradients(0)[:, 3, :].astype(np.float32))
        return (states, grads, res) if with_results else (states, grads)

    def hr_order(self, lr_results):
        """Queue order of the HR cases: with ``schedule='lr_longest_first'``
        the cases whose LR field still moved most at the end of the LR solve
        (largest last relative change) first, since the cases that settle
        slowest at LR are the ones that run longest at HR; a long case that
        starts early runs beside the short ones instead of alone at the end.
        ``'fifo'``: submission order. The order changes no case's result
        (every case's steps are independent of its slot), only the time."""
        n = len(lr_results)
        if self.schedule == "fifo":
            return np.arange(n)
        key = np.array([r["last_rel"] for r in lr_results], dtype=np.float64)
        key = np.where(np.isfinite(key), key, np.inf)
        return np.argsort(-key, kind="stable")

    def _hr_batch(self, s, machs, aoas, truth, inits, order, want_states=False, max_steps=None):
        """HR batch solve with the cases queued in `order`; results (and
        states) returned in the callers' case order."""
        order = np.asarray(order)
        if max_steps is not None and np.ndim(max_steps) > 0:
            max_steps = np.asarray(max_steps)[order]
        cases = self._cases(np.asarray(machs)[order], np.asarray(aoas)[order], np.asarray(truth)[order],
                            max_steps=max_steps)
        init_q = None if inits is None else [inits[i] for i in order]
        res_q, st_q = s.batch_solve(cases, init_fields=init_q, want_states=want_states)
        res, states = [None] * len(order), (None if st_q is None else [None] * len(order))
        for j, i in enumerate(order):
            res[i] = res_q[j]
            if st_q is not None:
                states[i] = st_q[j]
        return res, states

    def prepare(self, n_train=256, seed=3, target_steps=12000, train_steps=2000, batch=32768):
        """Training pairs from the batched solver (LR and HR solves of
        n_train cases drawn from default_rng(seed)), then the MLP trained by
        the library's BF16 kernels."""
        t0 = time.perf_counter()
        (mt, at), _ = draw_cases(n_train, 0, seed=seed)
        lr_states, lr_gp = self.lr_solutions(mt, at)
        self._solvers.pop(("lr", n_train)).close()
        hs = Solver(self.dm_hr, n_train, device=self.device, precision="f32", dt_mode="local",
                    stop_rule="reference", threshold=1e-30, check_every=self.check_every)
        _, hr_states = hs.batch_solve(self._cases(mt, at, max_steps=target_steps), want_states=True)
        hs.close()
        hr_gp = pressure_gradients(self.hr, self.dm_hr, hr_states, mt, at, device=self.device)
        data, mu, sig = build_training_set(self.ws, lr_states, lr_gp, hr_states, hr_gp, mt, at)
        del hr_states
        mlp = MLP(device=f"cuda:{self.device}", seed=0)
        self.ws.mlp = mlp
        loss_idw = eval_loss(None, data)
        hist, t_train = train(mlp, data, steps=train_steps, batch=batch)
        self.train_info = {"n_train": n_train, "rows": int(data.X.shape[0]), "target_steps": target_steps,
                           "train_steps": train_steps, "loss_idw": loss_idw, "loss_mlp": eval_loss(mlp, data),
                           "train_s": t_train, "setup_s": time.perf_counter() - t0}
        del data
        torch.cuda.empty_cache()
        return self.train_info

    def truth(self, machs, aoas, ref_steps=30000, confirm_steps=5000):
        """Reference CD of every case from a long float64 solve of the same
        kernels, and whether it is steady (CD moved by <= 0.1 % over the
        confirming steps)."""
        s = Solver(self.dm_hr, len(machs), precision="f64", dt_mode="local", stop_rule="reference",
                   threshold=1e-30, check_every=self.check_every, device=self.device)
        ra, states = s.batch_solve(self._cases(machs, aoas, max_steps=ref_steps, dtype=np.float64),
                                   want_states=True)
        rb, _ = s.batch_solve(self._cases(machs, aoas, max_steps=confirm_steps, dtype=np.float64),
                              init_fields=states)
        s.close()
        cd_a = np.array([r["cd"] for r in ra])
        cd = np.array([r["cd"] for r in rb])
        steady = np.abs(cd - cd_a) <= 1e-3 * np.abs(cd)
        return cd, steady

    def _hr_warm(self, s, machs, aoas, truth, inits, order, caps, want_states=False):
        """HR solve from the warm fields, case i capped at caps[i] steps. With
        a warm budget, a case the rule has not stopped within ``warm_budget``
        steps restarts from freestream with the rest of its cap (the plain
        start is the fallback: a prediction can leave the solve on another
        steady state, e.g. with a bow shock held at the LR mesh's stand-off).
        Its result carries ``fallback`` and the warm steps spent, counted in
        its ``steps`` and ``stopping_step``."""
        machs, aoas, truth = np.asarray(machs), np.asarray(aoas), np.asarray(truth)
        caps = np.asarray(caps, dtype=np.int64)
        budget = np.minimum(caps, self.warm_budget) if self.warm_budget else caps
        res, states = self._hr_batch(s, machs, aoas, truth, inits, order, want_states, max_steps=budget)
        if not self.warm_budget:
            return res, states
        rank = np.empty(len(order), dtype=np.int64)
        rank[np.asarray(order)] = np.arange(len(order))
        fb = np.array(sorted((i for i, r in enumerate(res) if r["status"] != 2 and caps[i] > int(r["steps"])),
                             key=lambda i: rank[i]), dtype=np.int64)
        if len(fb) == 0:
            return res, states
        spent_fb = np.array([int(res[i]["steps"]) for i in fb], dtype=np.int64)
        res2, st2 = self._hr_batch(s, machs[fb], aoas[fb], truth[fb], None, np.arange(len(fb)), want_states,
                                   max_steps=caps[fb] - spent_fb)
        for j, i in enumerate(fb):
            r = dict(res2[j])
            spent = int(res[i]["steps"])
            r["fallback"], r["warm_steps"] = True, spent
            r["steps"] = int(r["steps"]) + spent
            r["stopping_step"] = int(r["stopping_step"]) + spent
            res[i] = r
            if states is not None:
                states[i] = st2[j]
        return res, states

    # ----------------------------------------------------------- the stream
    def warm_fields(self, machs, aoas, use_mlp=True, parts=None):
        """LR solve, LR pressure gradients and the IDW (+ MLP) prediction of
        every case: the conserved HR warm fields (float64, HR cell order) and
        the HR queue order (``hr_order``)."""
        t = time.perf_counter()
        lr_states, lr_gp, lr_res = self.lr_solutions(machs, aoas, with_results=True)
        t1 = time.perf_counter()
        inits = [self.ws.predict_state(primitives(W).astype(np.float32), g, m, a, use_mlp=use_mlp)
                 for W, g, m, a in zip(lr_states, lr_gp, machs, aoas)]
        if parts is not None:
            parts["lr_solve_s"], parts["inference_s"] = t1 - t, time.perf_counter() - t1
        return inits, self.hr_order(lr_res)

    def solve_stream(self, batches, truth_of, steady_of, use_mlp=True):
        """Warm-started solves of a stream of case batches, as a campaign
        runs them: batch k+1's LR solve and prediction run while batch k's HR
        solve does (the HR batch is driven from a second host thread; each
        solver has its own stream, so the GPU runs both). batches: list of
        (machs, aoas); truth_of / steady_of: per-batch reference CDs and
        steady flags. Returns (per-batch PassResult, device seconds of the
        whole stream, wall seconds)."""
        import threading
        out = [None] * len(batches)
        s = self._hr_solver(min(self.slots, max(len(b[0]) for b in batches)))
        lo, hi = torch.cuda.Stream.priority_range()
        side = torch.cuda.Stream(device=self.device, priority=hi)   # the prediction's kernels, ahead of the HR chunks

        def hr(k, warm, box):
            try:
                torch.cuda.set_device(self.device)     # a new host thread starts on device 0
                m, a = batches[k]
                t = time.perf_counter()
                box["res"], _ = self._hr_warm(s, m, a, truth_of[k], *warm, self.caps(steady_of[k]))
                box["s"] = time.perf_counter() - t
            except BaseException as e:   # re-raised in the caller's thread
                box["err"] = e

        def run():
            warm = self.warm_fields(*batches[0], use_mlp=use_mlp)
            for k in range(len(batches)):
                box = {}
                th = threading.Thread(target=hr, args=(k, warm, box))
                th.start()
                t = time.perf_counter()
                nxt = None
                if k + 1 < len(batches):
                    side.wait_stream(torch.cuda.current_stream())
                    with torch.cuda.stream(side):
                        nxt = self.warm_fields(*batches[k + 1], use_mlp=use_mlp)
                    torch.cuda.current_stream().wait_stream(side)
                lr_s = time.perf_counter() - t
                th.join()
                if "err" in box:
                    raise box["err"]
                out[k] = self._score("mlp" if use_mlp else "idw", box["res"], truth_of[k], steady_of[k], 0.0, 0.0,
                                     {"hr_solve_s": box["s"], "next_lr_and_prediction_s": lr_s})
                warm = nxt
            return out

        _, sec, wall = _device_timed(run)
        return out, sec, wall

    # ------------------------------------------------------------- one pass
    def _score(self, start, res, truth, steady, seconds, wall, parts):
        st = np.array([r["status"] == 2 for r in res])
        cd = np.array([r["cd"] for r in res])
        ok = st & steady & (np.abs(cd - truth) <= self.cd_tol * np.abs(truth))
        return PassResult(start, res, int(ok.sum()), seconds, wall, parts,
                          [int(r["stopping_step"]) for r in res])

    def solve(self, machs, aoas, truth, steady, start="mlp", want_states=False):
        """One timed pass of `start` over the cases (see the module docstring)."""
        parts = {}

        def run():
            if start in ("cold", "single"):
                s = self._hr_solver(1 if start == "single" else min(self.slots, len(machs)))
                t = time.perf_counter()
                res, states = s.batch_solve(self._cases(machs, aoas, truth, max_steps=self.caps(steady)),
                                            want_states=want_states)
                parts["hr_solve_s"] = time.perf_counter() - t
                return res, states
            inits, order = self.warm_fields(machs, aoas, use_mlp=(start == "mlp"), parts=parts)
            s = self._hr_solver(min(self.slots, len(machs)))
            t = time.perf_counter()
            res, states = self._hr_warm(s, machs, aoas, truth, inits, order, self.caps(steady), want_states)
            parts["hr_solve_s"] = time.perf_counter() - t
            return res, states

        (res, states), sec, wall = _device_timed(run)
        out = self._score(start, res, truth, steady, sec, wall, parts)
        out.states = states
        return out
