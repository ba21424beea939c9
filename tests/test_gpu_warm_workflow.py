"""The warm-start workflow on the GPU: a stream of batches, whose next LR
solve and prediction run beside the current HR solve, gives every case the
result the one-batch-at-a-time pass gives it (eval/convergence_case.py:106-140
times the same pipeline one case set at a time)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wf():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from eulersr_b200.warmstart.workflow import WarmStartWorkflow
    w = WarmStartWorkflow(slots=4, lr_steps=800, max_steps=1500)
    w.prepare(n_train=8, target_steps=500, train_steps=20, batch=4096)
    yield w
    w.close()


def test_streamed_batches_equal_one_pass_each(wf):
    b1 = (np.array([0.50, 0.60, 0.70, 0.55, 0.65]), np.array([0.0, 1.0, 2.0, -1.0, 0.5]))
    b2 = (np.array([0.58, 0.68, 0.52]), np.array([1.5, -0.5, 2.5]))
    t1, s1 = wf.truth(*b1, ref_steps=2500, confirm_steps=500)
    t2, s2 = wf.truth(*b2, ref_steps=2500, confirm_steps=500)
    passes = [wf.solve(*b1, t1, s1, "mlp"), wf.solve(*b2, t2, s2, "mlp")]
    streamed, sec, wall = wf.solve_stream([b1, b2], [t1, t2], [s1, s2])
    assert sec > 0 and wall > 0
    for p, q in zip(passes, streamed):
        assert [r["stopping_step"] for r in p.results] == [r["stopping_step"] for r in q.results]
        assert [r["cd"] for r in p.results] == [r["cd"] for r in q.results]
        assert [r["status"] for r in p.results] == [r["status"] for r in q.results]
        assert p.converged == q.converged


def test_queue_order_changes_no_result(wf):
    m, a = np.array([0.50, 0.72, 0.60, 2.8, 0.65, 1.2]), np.array([0.0, 2.0, -1.0, 3.0, 1.0, -2.0])
    t, s = wf.truth(m, a, ref_steps=2500, confirm_steps=500)
    wf.schedule = "lr_longest_first"
    try:
        r_lpt = wf.solve(m, a, t, s, "mlp")
        r_lpt_st = wf.solve(m, a, t, s, "mlp", want_states=True)
    finally:
        wf.schedule = "fifo"
    r_fifo = wf.solve(m, a, t, s, "mlp", want_states=True)
    for key in ("stopping_step", "steps", "cd", "cl", "status"):
        assert [r[key] for r in r_lpt.results] == [r[key] for r in r_fifo.results], key
    for x, y in zip(r_fifo.states, r_lpt_st.states):
        assert np.array_equal(x, y)


def test_warm_budget_falls_back_to_freestream(wf):
    """A warm start the rule has not stopped within the warm budget restarts
    from freestream with the rest of the step cap: with a budget below the
    rule's 8 checks x 25 steps every case falls back, and each result is the
    freestream solve's under the remaining cap, with the warm steps added."""
    m, a = np.array([0.55, 2.2, 0.75]), np.array([1.0, -2.0, 3.0])
    t, s = wf.truth(m, a, ref_steps=2500, confirm_steps=500)
    budget, cap = wf.warm_budget, wf.max_steps
    wf.warm_budget = 100
    try:
        r = wf.solve(m, a, t, s, "mlp")
        wf.max_steps = cap - 100
        cold = wf.solve(m, a, t, s, "cold")
    finally:
        wf.warm_budget, wf.max_steps = budget, cap
    for x, y in zip(r.results, cold.results):
        assert x["fallback"] and x["warm_steps"] == 100
        assert x["steps"] == y["steps"] + 100 and x["stopping_step"] == y["stopping_step"] + 100
        assert (x["status"], x["cd"], x["cl"]) == (y["status"], y["cd"], y["cl"])


def test_unsteady_cap_stops_flagged_cases_for_every_start(wf):
    """With an unsteady cap, a case whose reference is flagged unsteady stops
    there for every start, and the other cases' results do not change."""
    m, a = np.array([0.6, 2.4, 0.7]), np.array([1.0, 2.0, -1.0])
    t, _ = wf.truth(m, a, ref_steps=2500, confirm_steps=500)
    flag = np.array([True, False, True])
    base = {st: wf.solve(m, a, t, flag, st) for st in ("mlp", "cold")}
    wf.unsteady_cap = 300
    try:
        capped = {st: wf.solve(m, a, t, flag, st) for st in ("mlp", "cold")}
    finally:
        wf.unsteady_cap = None
    for st in ("mlp", "cold"):
        r, b = capped[st].results, base[st].results
        assert r[1]["steps"] <= 300 and not r[1].get("fallback")
        for i in (0, 2):
            assert (r[i]["steps"], r[i]["cd"], r[i]["status"]) == (b[i]["steps"], b[i]["cd"], b[i]["status"])
