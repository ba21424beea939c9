"""CUDA kernels vs the NumPy oracle on the same meshes and inputs (the oracle
equals the reference's own solver source bit for bit, tests/
test_reference_fixtures.py), and directly vs that source's golden output.

Tolerances: float64 kernels vs float64 oracle 1e-12 (field-scaled relative,
after 100 SRK2 steps); float32 kernels vs float32 oracle 1e-5 after 100 steps
(the reference-fidelity mode; the fast mode is held to the reference float32's
own rounding band where a flow amplifies rounding, see its test);
force coefficients 1e-4 relative in float32. A whole float64 run (hundreds
of steps) is held to 1e-10. The float32 dt is held to 2e-6 relative: the oracle
derives the geometry in float32 as the reference does, the library derives it in
float64 and rounds once, so the minimum cell's area/perimeter term differs by
a few ulp.
"""
import numpy as np
import pytest

from conftest import oracle_mesh, rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def _oracle_steps(mesh, dtype, mach, aoa, steps, cfl=0.6, flux='hllc', recon='muscl', scheme='SRK2'):
    from oracle import euler_oracle as O
    om = oracle_mesh(mesh, dtype)
    cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=mach, aoa=aoa, case=mesh.metadata['case'])
    W, inlet = O.initialize(mesh.n_cells, cfg, dtype)
    c = 0.45 if (0.6 < mach < 1.1 and cfl > 0.45) else cfl
    dt = O.get_dt(W, om, CFL=c)
    fn = O.TIME_SCHEMES[scheme]
    for _ in range(steps):
        W = fn(W, om, dt, inlet, reconstruction=recon, flux=flux)
    return W, dt, om, inlet


def _gpu_steps(mesh, prec, mach, aoa, steps, cfl=0.6, flux='hllc', recon='muscl', scheme='SRK2', **kw):
    from eulersr_b200.solver import Solver, FlowCase
    dtype = np.float64 if prec == 'f64' else np.float32
    s = Solver(mesh, 1, precision=prec, flux=flux, reconstruction=recon, time_scheme=scheme, **kw)
    s.set_case(0, FlowCase(mach=mach, aoa_deg=aoa, cfl=cfl, tf=100.0, dtype=dtype, l_ref=1.0))
    dt = s.dt()[0]
    s.step(steps)
    W = s.get_state(0)
    return W, dt, s


@pytest.mark.parametrize("prec,fidelity,tol", [("f64", "fast", TOL64), ("f32", "reference", TOL32)])
def test_srk2_100_steps_diamond(diamond02, prec, fidelity, tol):
    dtype = np.float64 if prec == 'f64' else np.float32
    Wo, dto, _, _ = _oracle_steps(diamond02, dtype, 2.5, 5.0, 100)
    Wg, dtg, _ = _gpu_steps(diamond02, prec, 2.5, 5.0, 100, fidelity=fidelity)
    dt_tol = 1e-14 if prec == 'f64' else 2e-6
    assert abs(dtg - float(dto)) <= dt_tol * float(dto)
    print(f"diamond h=0.2 {prec} {fidelity}: {rel_err(Wg, Wo):.3e} after 100 steps")
    assert rel_err(Wg, Wo) <= tol, rel_err(Wg, Wo)


def test_srk2_100_steps_diamond_fast_f32(diamond02):
    """The fast float32 mode (geometry from float64 rounded once, approximate
    divides, each face's flux from its owner) rounds differently from the
    reference's float32, and this flow amplifies rounding: the reference's own
    float32 ends 1.2e-5 from the float64 solution of the same scheme here, and
    one half-ulp perturbation of its state after the first step moves it by
    0.5-0.8e-5 after 100 steps. So the fast mode is held to that band: within
    twice the reference float32's own distance from float64 of the reference's
    float32, and no further from float64 than 1.5 times that distance (at
    least as accurate as the reference's float32). The reference-fidelity mode
    is the 1e-5 parity mode (above)."""
    Wo32, dto, _, _ = _oracle_steps(diamond02, np.float32, 2.5, 5.0, 100)
    Wo64, _, _, _ = _oracle_steps(diamond02, np.float64, 2.5, 5.0, 100)
    Wg, dtg, _ = _gpu_steps(diamond02, 'f32', 2.5, 5.0, 100, fidelity='fast')
    assert abs(dtg - float(dto)) <= 2e-6 * float(dto)
    band = rel_err(Wo32, Wo64)
    e_ref, e_64 = rel_err(Wg, Wo32), rel_err(Wg, Wo64)
    print(f"diamond h=0.2 f32 fast: {e_ref:.3e} from the reference float32, {e_64:.3e} from float64 "
          f"(reference float32 from float64: {band:.3e})")
    assert e_ref <= 2.0 * band, (e_ref, band)
    assert e_64 <= 1.5 * band, (e_64, band)


def test_srk2_transonic_naca_f64(naca02):
    Wo, dto, _, _ = _oracle_steps(naca02, np.float64, 0.8, 2.0, 60)
    Wg, dtg, _ = _gpu_steps(naca02, 'f64', 0.8, 2.0, 60)
    assert abs(dtg - dto) <= 1e-14 * dto
    assert rel_err(Wg, Wo) <= TOL64


@pytest.mark.parametrize("flux,recon,scheme", [("rusanov", "muscl", "SRK2"), ("hllc", "constant", "SRK2"),
                                               ("hllc", "muscl", "EE"), ("hllc", "muscl", "RK2"),
                                               ("rusanov", "constant", "EE")])
def test_scheme_variants_f64(diamond02, flux, recon, scheme):
    Wo, _, _, _ = _oracle_steps(diamond02, np.float64, 1.8, -3.0, 30, flux=flux, recon=recon, scheme=scheme)
    Wg, _, _ = _gpu_steps(diamond02, 'f64', 1.8, -3.0, 30, flux=flux, recon=recon, scheme=scheme)
    assert rel_err(Wg, Wo) <= TOL64


def test_golden_fixture_f64(diamond02, golden):
    g = np.load(golden / "oracle_diamond_h0.2_M2.5_a5_srk2x20.npz")
    Wg, dtg, _ = _gpu_steps(diamond02, 'f64', 2.5, 5.0, int(g['steps']))
    assert abs(dtg - float(g['dt'])) <= 1e-14 * float(g['dt'])
    assert rel_err(Wg, g['W']) <= TOL64


def test_forces_entropy_probe(diamond02):
    from oracle import euler_oracle as O
    Wo, dto, om, inlet = _oracle_steps(diamond02, np.float64, 2.0, 0.0, 50)
    Wg, _, s = _gpu_steps(diamond02, 'f64', 2.0, 0.0, 50)
    cd, cl = s.forces()
    cdo, clo = O.force_coefficients(Wo, om, 1.0, 2.0 * np.sqrt(1.4), 1.0)
    assert abs(cd[0] - cdo) <= 1e-10 * max(abs(cdo), 1e-3)
    assert abs(cl[0] - clo) <= 1e-10 + 1e-10 * abs(clo)
    S = s.entropy()[0]
    So = O.total_entropy(Wo, om, 1.4)
    assert abs(S - So) <= 1e-10 * max(1.0, abs(So))
    rel = s.residual_probe()[0]
    Wp = O.time_step_srk2(Wo, om, dto, inlet)
    relo = np.linalg.norm(Wp - Wo) / (np.linalg.norm(Wo) + 1e-16)
    assert abs(rel - relo) <= 1e-8 * relo
    # the probe must not change the state
    assert np.array_equal(s.get_state(0), Wg)


def test_determinism_and_graphs(diamond02):
    Wa, _, _ = _gpu_steps(diamond02, 'f32', 2.5, 5.0, 40, use_graphs=True)
    Wb, _, _ = _gpu_steps(diamond02, 'f32', 2.5, 5.0, 40, use_graphs=True)
    Wc, _, _ = _gpu_steps(diamond02, 'f32', 2.5, 5.0, 40, use_graphs=False)
    assert np.array_equal(Wa, Wb)
    assert np.array_equal(Wa, Wc)


def test_renumbering_invariance(diamond02):
    from eulersr_b200.solver import Solver, FlowCase, DeviceMesh
    out = []
    for ren in (True, False):
        s = Solver(DeviceMesh(diamond02, renumber=ren), 1, precision='f64')
        s.set_case(0, FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.6, tf=100.0))
        s.step(30)
        out.append(s.get_state(0))
    assert np.array_equal(out[0], out[1])


def test_stop_rule_matches_oracle_f64(diamond02):
    """Full run with the reference stop rule: same stopping step, converged flag
    and final field as the oracle's loop (euler/main.py:141-216)."""
    from oracle import euler_oracle as O
    from eulersr_b200.solver import Solver, FlowCase
    cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0, case='diamond', CFL=0.6, tf=6.0,
               stationarity_threshold=1e-4, stationarity_check_every=25, stationarity_patience=2)
    om = oracle_mesh(diamond02, np.float64)
    W0, inlet = O.initialize(diamond02.n_cells, cfg, np.float64)
    ro = O.run(W0, om, inlet, cfg)
    s = Solver(diamond02, 1, precision='f64', threshold=1e-4, check_every=25, patience=2)
    s.set_case(0, FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.6, tf=6.0))
    r = s.run()[0]
    assert r['n_max'] == ro.n_max
    assert bool(r['converged']) == ro.converged
    assert r['stopping_step'] == ro.stopping_step
    assert rel_err(s.get_state(0), ro.W) <= 1e-10


def test_maxstep_cap(diamond02):
    from eulersr_b200.solver import Solver, FlowCase
    s = Solver(diamond02, 1, precision='f32', threshold=1e-30, check_every=7)
    s.set_case(0, FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.6, tf=0.05))
    r = s.run()[0]
    assert r['status'] == 3 and not r['converged']
    assert r['steps'] == r['n_max'] == int(np.float32(0.05) / np.float32(r['dt'])) + 1


@pytest.mark.parametrize("precision,block", [("f32", 0), ("f32", "patches"), ("f64", 0)])
def test_batch_equals_single(diamond02, naca02, precision, block):
    """Every case solved inside a ragged two-mesh batch, with the queue
    retiring and refilling slots on the device, is bitwise identical to the
    same case solved alone: state, stop step, status and force coefficients.
    Case 4 starts from a warm field and case 1 tracks the engineering rule.
    With block='patches' the batch's K2 runs by patches (face fluxes once per
    inner face) while the single solves run the per-cell K2."""
    from eulersr_b200.solver import Solver, FlowCase
    dt_ = np.float32 if precision == 'f32' else np.float64
    meshes = [diamond02, naca02]
    spec = [(2.5, 5.0), (1.5, -2.0), (3.0, 1.0), (0.9, 0.5), (2.0, 0.0), (2.2, 3.0), (1.8, -1.0)]
    cases = [FlowCase(mach=m, aoa_deg=a, mesh=i % 2, cfl=0.6, tf=0.4, dtype=dt_) for i, (m, a) in enumerate(spec)]
    eng = dict(eng_target_cd=0.05, eng_target_cl=0.1, eng_cd_tol=0.5, eng_cl_tol=100.0, eng_patience=2)
    for k, v in eng.items():
        setattr(cases[1], k, v)
    warm = Solver(diamond02, 1, precision=precision)
    warm.set_case(0, FlowCase(mach=2.0, aoa_deg=0.0, cfl=0.6, tf=0.4, dtype=dt_))
    warm.step(30)
    init = [None] * len(cases)
    init[4] = warm.get_state(0)
    s = Solver(meshes, [2, 1], precision=precision, threshold=1e-5, check_every=10, block_size=block)
    res, states = s.batch_solve(cases, init_fields=init, want_states=True)
    assert sorted(r['case_index'] for r in res) == list(range(len(cases)))
    for i, c in enumerate(cases):
        one = Solver(meshes[c.mesh], 1, precision=precision, threshold=1e-5, check_every=10, block_size=128)
        c1 = FlowCase(mach=c.mach, aoa_deg=c.aoa_deg, cfl=0.6, tf=0.4, dtype=dt_)
        if i == 1:
            for k, v in eng.items():
                setattr(c1, k, v)
        one.set_case(0, c1, init[i])
        r1 = one.run()[0]
        for k in ('stopping_step', 'status', 'steps', 'n_max', 'cd', 'cl', 'eng_converged', 'eng_stopping_step'):
            assert r1[k] == res[i][k], (i, k, r1[k], res[i][k])
        assert np.array_equal(one.get_state(0), states[i]), i
        # the probe of the retiring case (euler/main.py:228-230) with the case's own dt
        assert res[i]['final_residual'] == one.residual_probe()[0], i
    # the same batch again on the same handle gives the same answer
    res2, states2 = s.batch_solve(cases, init_fields=init, want_states=True)
    assert all(np.array_equal(a, b) for a, b in zip(states, states2))
    assert [r['stopping_step'] for r in res] == [r['stopping_step'] for r in res2]


def test_batch_submit_poll_results(diamond02, naca02):
    """esr_batch_submit / esr_batch_poll / esr_batch_results give bitwise the
    results and final states of esr_batch_solve. While a batch owns the slots
    other solver calls fail with ESR_ERR_STATE; results before the end fail;
    a cancelled batch leaves the solver usable for the next batch."""
    from eulersr_b200.solver import Solver, FlowCase
    from eulersr_b200._ffi import EsrError
    meshes = [diamond02, naca02]
    spec = [(2.5, 5.0), (1.5, -2.0), (3.0, 1.0), (0.9, 0.5), (2.0, 0.0), (2.2, 3.0), (1.8, -1.0)]
    cases = [FlowCase(mach=m, aoa_deg=a, mesh=i % 2, cfl=0.6, tf=0.4, dtype=np.float32)
             for i, (m, a) in enumerate(spec)]
    warm = Solver(diamond02, 1, precision='f32')
    warm.set_case(0, FlowCase(mach=2.0, aoa_deg=0.0, cfl=0.6, tf=0.4, dtype=np.float32))
    warm.step(30)
    init = [None] * len(cases)
    init[4] = warm.get_state(0)
    s = Solver(meshes, [2, 1], precision='f32', threshold=1e-5, check_every=10)
    ref, ref_states = s.batch_solve(cases, init_fields=init, want_states=True)
    s.batch_submit(cases, init_fields=init, want_states=True)
    with pytest.raises(EsrError):
        s.step(1)
    with pytest.raises(EsrError):
        s.batch_submit(cases)
    with pytest.raises(EsrError):
        s.batch_results()
    done, polls, seen = 0, 0, []
    while done < len(cases):
        done = s.batch_poll()
        seen.append(done)
        polls += 1
        assert polls < 100000
    assert seen == sorted(seen)
    res, states = s.batch_results()
    for k in ('stopping_step', 'status', 'steps', 'n_max', 'cd', 'cl', 'final_residual', 'case_index'):
        assert [r[k] for r in res] == [r[k] for r in ref], k
    assert all(np.array_equal(a, b) for a, b in zip(states, ref_states))
    # cancel part-way, then the solver takes the next batch and single cases again
    s.batch_submit(cases, init_fields=init)
    s.batch_poll()
    s.batch_cancel()
    res3, _ = s.batch_solve(cases, init_fields=init)
    assert [r['stopping_step'] for r in res3] == [r['stopping_step'] for r in ref]
    s.set_case(0, cases[0])
    s.step(2)
    # an empty batch: nothing runs, the slots are left as they are
    s.batch_submit([])
    assert s.batch_poll() == 0
    assert s.batch_results() == ([], None)


def test_autotuner_and_block_invariance(naca02):
    """The autotuner times every launch shape (cell kernels at 64, 128 and
    256 threads, K2's second register budget, K2 by patches at both budgets,
    K1's second budget) and keeps the fastest; a second solver of the same
    shape takes the choice from the process cache. The state after 30 steps
    is bitwise the same whatever the shape: K2 by patches evaluates each inner
    face once and the per-cell K2 the same canonical flux from the face's
    owner, with explicit rounding in both, so neither the kernel form nor the
    register budget changes a bit."""
    from eulersr_b200.solver import Solver, FlowCase

    def run(s):
        for g, (m, a) in enumerate([(0.8, 1.0), (2.0, -3.0), (1.3, 2.5)]):
            s.set_case(g, FlowCase(mach=m, aoa_deg=a, tf=1.0, dtype=np.float32))
        s.step(30)
        return [s.get_state(g) for g in range(3)]

    states = []
    s = Solver(naca02, 3, precision='f32', block_size=0)
    t = s.tuning()
    assert sorted(t['step_ms'], key=str) == [128, 256, 64, "patches"]
    assert all(v > 0 for v in t['step_ms'].values())
    var = t['variants']
    assert len(var) == 7 and all(v['step_ms'] > 0 for v in var)
    assert [v['block_size'] for v in var[:3]] == [64, 128, 256]
    assert {(v['k2_patches'], v['k2_minb']) for v in var} == {(False, 5), (False, 4), (True, 5), (True, 6)}
    assert {v['k1_minb'] for v in var} == {8, 6}
    best = min(var, key=lambda v: v['step_ms'])
    assert (t['block_size'], t['k2_patches'], t['k1_minb'], t['k2_minb']) == (
        best['block_size'], best['k2_patches'], best['k1_minb'], best['k2_minb'])
    states.append(run(s))
    again = Solver(naca02, 3, precision='f32', block_size=0)
    t2 = again.tuning()
    assert t2['cached'] and t2['variants'] == var and t2['block_size'] == t['block_size']
    # every timed shape, set by hand
    for v in var:
        s.set_shape(v['block_size'], v['k2_patches'], v['k1_minb'], v['k2_minb'])
        got = s.tuning()
        assert (got['block_size'], got['k2_patches'], got['k1_minb'], got['k2_minb']) == (
            v['block_size'], v['k2_patches'], v['k1_minb'], v['k2_minb'])
        states.append(run(s))
    for bs in (64, 128, 256, "patches"):
        s = Solver(naca02, 3, precision='f32', block_size=bs)
        t = s.tuning()
        if bs == "patches":
            assert t['k2_patches'] and t['block_size'] == 128 and t['step_ms'] == {}
        else:
            assert t['block_size'] == bs and not t['k2_patches'] and t['step_ms'] == {}
        states.append(run(s))
    for other in states[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(states[0], other))
    # shapes a solver cannot run are refused
    from eulersr_b200._ffi import EsrError
    f64 = Solver(naca02, 1, precision='f64', block_size=64)
    with pytest.raises(EsrError):
        f64.set_shape(64, True)
    with pytest.raises(EsrError):
        f64.set_shape(64, False, 0, 4)
    with pytest.raises(EsrError):
        s.set_shape(96)
    with pytest.raises(EsrError):
        s.set_shape(64, False, 7, 0)
    # a submitted batch owns the slots: the shape cannot change under it
    s.batch_submit([FlowCase(mach=1.5, aoa_deg=1.0, tf=0.2, max_steps=40, dtype=np.float32)])
    with pytest.raises(EsrError):
        s.set_shape(128)
    while s.batch_poll() < 1:
        pass
    res, _ = s.batch_results()
    assert len(res) == 1
    s.set_shape(128)


def test_set_cases_get_states_match_per_slot_calls(diamond02, naca02):
    """esr_set_cases / esr_get_states (many slots, one synchronisation) give
    bitwise the same runs as esr_set_case / esr_get_state slot by slot, on a
    two-mesh solver with warm-started and freestream slots."""
    from eulersr_b200.solver import Solver, FlowCase
    meshes = [diamond02, naca02]
    spec = [(0, 2.5, 5.0), (0, 1.5, -2.0), (1, 0.9, 1.0), (1, 2.0, 0.0), (1, 3.0, -4.0)]
    cases = [FlowCase(mach=m, aoa_deg=a, mesh=k, cfl=0.6, tf=0.5, dtype=np.float32) for k, m, a in spec]
    slots = [0, 1, 2, 3, 4]
    pre = Solver(naca02, 1, precision='f32')
    pre.set_case(0, FlowCase(mach=2.0, aoa_deg=0.0, tf=0.5, dtype=np.float32))
    pre.step(15)
    warm = [None, None, None, pre.get_state(0), None]
    a = Solver(meshes, [2, 3], precision='f32', threshold=1e-5, check_every=10)
    b = Solver(meshes, [2, 3], precision='f32', threshold=1e-5, check_every=10)
    for g, c, w in zip(slots, cases, warm):
        a.set_case(g, c, w)
    b.set_cases(slots[::-1], cases[::-1], warm[::-1])
    assert np.array_equal(a.dt(), b.dt())
    a.step(40)
    b.step(40)
    got = b.get_states(slots)
    for g in slots:
        assert np.array_equal(a.get_state(g), got[g]), g
    ra, rb = a.run(), b.run()
    assert [r['stopping_step'] for r in ra] == [r['stopping_step'] for r in rb]
    assert [r['case_index'] for r in ra] == [r['case_index'] for r in rb] == slots
    with pytest.raises(Exception):
        b.set_cases([0, 0], cases[:2])
    # a call with an invalid case changes nothing, not even the valid slots before it
    before = b.get_states(slots)
    bad = FlowCase(mach=2.0, aoa_deg=0.0, mesh=1, cfl=-1.0, tf=0.5, dtype=np.float32)
    with pytest.raises(Exception):
        b.set_cases([0, 2], [cases[0], bad])
    after = b.get_states(slots)
    for g in slots:
        assert np.array_equal(before[g], after[g]), g
    # float32 host fields: the float32 solver stores exactly the same values
    c32 = Solver(meshes, [2, 3], precision='f32', threshold=1e-5, check_every=10)
    warm32 = [None if w is None else w.astype(np.float32) for w in warm]
    c32.set_cases(slots, cases, warm32)
    c32.step(40)
    got32 = c32.get_states(slots, dtype=np.float32)
    for g in slots:
        assert got32[g].dtype == np.float32
        assert np.array_equal(got32[g], got[g].astype(np.float32)), g


def test_set_cases_get_states_float64_solver(diamond02, naca02):
    """The batched transfers on a float64 solver (two meshes, warm and
    freestream slots) equal the per-slot calls bitwise; float32 host fields
    are widened exactly."""
    from eulersr_b200.solver import Solver, FlowCase
    meshes = [diamond02, naca02]
    spec = [(0, 2.5, 5.0), (1, 0.9, 1.0), (1, 2.0, 0.0)]
    cases = [FlowCase(mach=m, aoa_deg=a, mesh=k, cfl=0.6, tf=0.5) for k, m, a in spec]
    slots = [0, 1, 2]
    rng = np.random.default_rng(7)
    warm = [None, None, np.tile(cases[2].to_c().inlet[:], (naca02.n_cells, 1))
            * (1.0 + 0.01 * rng.standard_normal((naca02.n_cells, 1)))]
    a = Solver(meshes, [1, 2], precision='f64', threshold=1e-5, check_every=10)
    b = Solver(meshes, [1, 2], precision='f64', threshold=1e-5, check_every=10)
    for g, c, w in zip(slots, cases, warm):
        a.set_case(g, c, w)
    b.set_cases(slots, cases, warm)
    assert np.array_equal(a.dt(), b.dt())
    a.step(20)
    b.step(20)
    got = b.get_states(slots)
    for g in slots:
        assert got[g].dtype == np.float64
        assert np.array_equal(a.get_state(g), got[g]), g
    w32 = [None, None, warm[2].astype(np.float32)]
    c = Solver(meshes, [1, 2], precision='f64', threshold=1e-5, check_every=10)
    c.set_cases(slots, cases, w32)
    d = Solver(meshes, [1, 2], precision='f64', threshold=1e-5, check_every=10)
    d.set_cases(slots, cases, [None, None, w32[2].astype(np.float64)])
    assert all(np.array_equal(x, y) for x, y in zip(c.get_states(slots), d.get_states(slots)))


def test_batch_edge_cases(diamond02):
    """Queue edge cases of esr_batch_solve: an empty case list, a case capped
    by max_steps (MAXSTEP), a case that blows up (CFL 40: NONFINITE, retired
    at its next check without disturbing the others), and more cases than
    slots on one slot; every finite case equals its single-case solve."""
    from eulersr_b200.solver import Solver, FlowCase
    s = Solver(diamond02, 1, precision='f32', threshold=1e-5, check_every=10)
    res, states = s.batch_solve([], want_states=True)
    assert res == [] and states == []
    cases = [FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.6, tf=10.0, max_steps=7, dtype=np.float32),
             FlowCase(mach=2.0, aoa_deg=1.0, cfl=40.0, tf=10.0, max_steps=400, dtype=np.float32),
             FlowCase(mach=1.5, aoa_deg=-1.0, cfl=0.6, tf=0.3, dtype=np.float32)]
    res, states = s.batch_solve(cases, want_states=True)
    assert res[0]['status'] == 3 and res[0]['steps'] == 7 and res[0]['n_max'] == 7
    assert res[1]['status'] == 4 and not res[1]['converged']
    assert res[2]['status'] in (2, 3)
    for i in (0, 2):
        one = Solver(diamond02, 1, precision='f32', threshold=1e-5, check_every=10)
        one.set_case(0, cases[i])
        r1 = one.run()[0]
        assert r1['stopping_step'] == res[i]['stopping_step'] and r1['status'] == res[i]['status']
        assert np.array_equal(one.get_state(0), states[i])


def test_per_case_threshold(diamond02):
    """esr_case.threshold overrides the solver's stop-rule threshold for that
    case (batch and single-slot paths alike), as eval/convergence_case.py
    gives each case its own."""
    from eulersr_b200.solver import Solver, FlowCase
    thr = [3e-4, 5e-5, None]
    cases = [FlowCase(mach=2.0, aoa_deg=2.0, cfl=0.6, tf=2.0, threshold=t, dtype=np.float32) for t in thr]
    s = Solver(diamond02, 2, precision='f32', threshold=1e-3, check_every=10, patience=2)
    res, _ = s.batch_solve(cases)
    for c, t, r in zip(cases, thr, res):
        one = Solver(diamond02, 1, precision='f32', threshold=t if t is not None else 1e-3, check_every=10,
                     patience=2)
        one.set_case(0, FlowCase(mach=2.0, aoa_deg=2.0, cfl=0.6, tf=2.0, dtype=np.float32))
        r1 = one.run()[0]
        assert (r1['stopping_step'], r1['status']) == (r['stopping_step'], r['status']), (t, r1, r)
    assert res[1]['stopping_step'] > res[0]['stopping_step'] > res[2]['stopping_step']


@pytest.mark.parametrize("tag,name,mach,aoa,prec,fidelity,tol", [
    ("diamond", "diamond_h0.2", 2.5, 5.0, "f64", "fast", 1e-12),
    ("naca", "naca0012_h0.2", 0.8, 1.25, "f64", "fast", 1e-12),
    ("diamond", "diamond_h0.2", 2.5, 5.0, "f32", "fast", 1e-5),
    ("diamond", "diamond_h0.2", 2.5, 5.0, "f32", "reference", 1e-5),
    ("naca", "naca0012_h0.2", 0.8, 1.25, "f32", "reference", 1e-5)])
def test_cuda_against_reference_solver_source(tag, name, mach, aoa, prec, fidelity, tol):
    """The CUDA path against EulerSR's own solver source run with NumPy for
    jax.numpy (tests/golden/reference_solver.npz, made by
    tests/golden/make_reference_fixtures.py): 20 SRK2 steps and the dt. With
    the reference fidelity the float32 dt is the reference's bit for bit."""
    from conftest import GOLDEN, load_mesh
    ref = np.load(GOLDEN / "reference_solver.npz")
    Wg, dtg, _ = _gpu_steps(load_mesh(name), prec, mach, aoa, 20, fidelity=fidelity)
    dt_ref = float(ref[f"{tag}_{prec}_dt"])
    if fidelity == "reference":
        assert dtg == dt_ref
    assert abs(dtg - dt_ref) <= (1e-14 if prec == "f64" else 2e-6) * dt_ref
    err = rel_err(Wg, ref[f"{tag}_{prec}_W20"])
    print(f"{name} {prec} {fidelity}: {err:.3e} after 20 steps")
    assert err <= tol


@pytest.mark.parametrize("layout", ["separate", "one_block"])
def test_overlapped_transfers_equal_synchronous(diamond02, naca02, layout):
    """The pipelined form of set_cases / step / get_states (next cases staged
    on the copy stream while the current chunk runs, final fields fetched
    while the next runs) gives bitwise the fields of the synchronous calls,
    over three rounds of different warm fields on a two-mesh solver; with
    every field a view of one host block ('one_block') the library moves
    them with one copy each way, with separate arrays one per case."""
    import torch
    from eulersr_b200.solver import Solver, FlowCase, freestream
    meshes = [diamond02, naca02]
    spec = [(0, 2.5, 5.0), (0, 1.5, -2.0), (1, 0.9, 1.0), (1, 2.0, 0.0)]
    cases = [FlowCase(mach=m, aoa_deg=a, mesh=k, cfl=0.6, tf=1e9, dtype=np.float32) for k, m, a in spec]
    slots = [0, 1, 2, 3]
    rng = np.random.default_rng(5)
    sizes = [meshes[c.mesh].n_cells for c in cases]

    def host_arrays():
        if layout == "separate":
            return [torch.empty((n, 4), dtype=torch.float32, pin_memory=True).numpy() for n in sizes]
        big = torch.empty((sum(sizes), 4), dtype=torch.float32, pin_memory=True).numpy()
        offs = np.concatenate([[0], np.cumsum(sizes)])
        return [big[offs[i]:offs[i + 1]] for i in range(len(sizes))]

    rounds = []
    for r in range(3):
        fields = host_arrays()
        for c, pinned in zip(cases, fields):
            n = meshes[c.mesh].n_cells
            W = np.repeat(freestream(c.mach, c.aoa_deg, dtype=np.float32)[None, :], n, 0)
            pinned[:] = (W * (1 + 0.01 * r * rng.standard_normal((n, 1)))).astype(np.float32)
        rounds.append(fields)
    sync = Solver(meshes, [2, 2], precision="f32", block_size=128)
    want = []
    for fields in rounds:
        sync.set_cases(slots, cases, fields)
        sync.step(20)
        want.append(sync.get_states(slots, dtype=np.float32))
    pipe = Solver(meshes, [2, 2], precision="f32", block_size=128)
    outs = [host_arrays() for _ in rounds]
    pipe.stage_cases(slots, cases, rounds[0])
    pipe.apply_staged()
    for r in range(3):
        if r + 1 < 3:
            pipe.stage_cases(slots, cases, rounds[r + 1])
        pipe.step(20)
        pipe.fetch_states(slots, outs[r])
        if r + 1 < 3:
            pipe.apply_staged()
    pipe.wait_transfers()
    for r in range(3):
        for a, b in zip(outs[r], want[r]):
            assert np.array_equal(a, b), r
    with pytest.raises(Exception):
        pipe.apply_staged()      # nothing staged
    sync.close()
    pipe.close()


def test_solver_refuses_cells_times_slots_beyond_2_31(diamond02):
    """The item index of a mesh (cell x slots + slot) is 32-bit in the
    kernels: a solver whose cells x slots reach 2^31 is refused with
    ESR_ERR_ARG at creation, before its state arrays are allocated."""
    from eulersr_b200._ffi import EsrError
    from eulersr_b200.solver import Solver
    n = diamond02.n_cells
    slots = (2 ** 31 + n - 1) // n           # n * slots >= 2^31
    with pytest.raises(EsrError) as e:
        Solver(diamond02, slots, precision='f32', block_size=128)
    assert e.value.code == 1 and "2^31" in str(e.value)
