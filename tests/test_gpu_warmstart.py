"""The learned warm start end to end at a small size (NACA2412, HR h=0.1,
LR h=0.2): the batched solver produces the training fields, the library's
kernels train the MLP, and on held-out cases the trained network's initial
field is closer to the converged HR solution than IDW alone, and the FVM
started from it reaches the reference CD in fewer iterations than from
freestream."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_warm_start_gains_over_idw_and_freestream():
    from eulersr_b200.meshing import build_mesh
    from eulersr_b200.solver import DeviceMesh
    from eulersr_b200.warmstart.features import MeshPair
    from eulersr_b200.warmstart.mlp import MLP
    from eulersr_b200.warmstart.pipeline import (WarmStart, build_training_set, draw_cases, pressure_gradients,
                                                 primitives, train)
    from eulersr_b200.warmstart.run import solve
    hr, lr = build_mesh("naca2412", 0.1), build_mesh("naca2412", 0.2)
    pair = MeshPair.build(hr, lr)
    dm_hr, dm_lr = DeviceMesh(hr), DeviceMesh(lr)
    nt, ne = 64, 12
    (mt, at), (me, ae) = draw_cases(nt, ne, seed=5)
    ma, aa = np.r_[mt, me], np.r_[at, ae]
    _, lr_states, _ = solve(dm_lr, ma, aa, max_steps=3000, want_states=True)
    lr_gp = pressure_gradients(lr, dm_lr, lr_states, ma, aa)
    _, hr_states, _ = solve(dm_hr, mt, at, max_steps=6000, want_states=True)
    hr_gp = pressure_gradients(hr, dm_hr, hr_states, mt, at)
    ws = WarmStart(pair)
    data, _, _ = build_training_set(ws, lr_states[:nt], lr_gp[:nt], hr_states, hr_gp, mt, at)
    mlp = MLP(seed=0)
    ws.mlp = mlp
    train(mlp, data, steps=600, batch=8192)
    ref, ref_states, _ = solve(dm_hr, me, ae, max_steps=6000, want_states=True)
    inits, err = {}, {}
    for use in (False, True):
        fields, e = [], []
        for i in range(ne):
            W0 = ws.predict_state(primitives(lr_states[nt + i]).astype(np.float32), lr_gp[nt + i], me[i], ae[i],
                                  use_mlp=use)
            fields.append(W0)
            P0, Pr = primitives(W0), primitives(ref_states[i])
            e.append(np.linalg.norm(P0 - Pr) / np.linalg.norm(Pr))
        inits[use], err[use] = fields, float(np.median(e))
    assert err[True] < 0.9 * err[False], err
    truth = [r["cd"] for r in ref]
    kw = dict(stop_rule="engineering", max_steps=6000, cd_targets=truth, cd_tol=0.01, patience=4)
    cold, _, _ = solve(dm_hr, me, ae, **kw)
    warm, _, _ = solve(dm_hr, me, ae, init_fields=inits[True], **kw)
    it_cold = np.median([r["stopping_step"] for r in cold])
    it_warm = np.median([r["stopping_step"] for r in warm])
    assert it_warm < 0.8 * it_cold, (it_warm, it_cold)
