"""Drop-in entry points on the GPU: euler/main.py run(), the eval worker
protocol, the engineering criterion, the density-L2 and local-dt options, the
gradient export, the subsonic-inlet boundary, and the analytic diamond
validation (shock-expansion theory)."""
import json
import math
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, oracle_mesh, rel_err

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    from eulersr_b200.config import load_default_config
    cfg = load_default_config()
    cfg.update(case='diamond', Mach=2.5, aoa=5.0, CFL=0.6, tf=6.0, stationarity_threshold=1e-4,
               stationarity_check_every=25, stationarity_patience=2, precision='f64', verbose=True)
    cfg['export'] = dict(results=False, figures=False, graph=False, summary=True, bundle=True, n_snaps=1)
    cfg.update(kw)
    return cfg


def test_main_run_matches_oracle(diamond02, tmp_path, capsys):
    from eulersr_b200 import main as M
    from oracle import euler_oracle as O
    cfg = _cfg()
    W0, inlet = M.initialize(diamond02, cfg)
    out = {'fig': tmp_path / 'fig', 'res': tmp_path / 'res'}
    W = M.run(W0, diamond02, inlet, dict(cfg), out)
    text = capsys.readouterr().out
    import re
    m = re.search(r'Simulation termin.+? en ([\d.]+)s \(converged=(True|False), t=([\d.]+)s\)', text)
    assert m, text
    om = oracle_mesh(diamond02, np.float64)
    Wo, inl = O.initialize(diamond02.n_cells, cfg)
    ro = O.run(Wo, om, inl, dict(cfg))
    assert (m.group(2) == 'True') == ro.converged
    assert rel_err(W, ro.W) <= 1e-10
    summ = json.loads(next((tmp_path / 'res').glob('summary_*.json')).read_text())
    for k in ("case", "h", "n_cells", "cd", "cl", "deltaS", "stationarity_rel", "converged", "stopping_step",
              "stationarity_threshold", "stationarity_check_every", "stationarity_patience", "wall_time_s",
              "compile_time_s", "solve_time_s", "engineering_converged", "engineering_stopping_step",
              "engineering_target_cd", "engineering_target_cl", "time_scheme", "flux", "reconstruction", "mach",
              "mesh_path", "aoa"):
        assert k in summ
    assert summ['stopping_step'] == ro.stopping_step
    cd, cl = O.force_coefficients(ro.W, om, 1.0, 2.5 * math.sqrt(1.4), 1.0)
    assert summ['cd'] == pytest.approx(cd, rel=1e-9) and summ['cl'] == pytest.approx(cl, rel=1e-9)
    dS = O.total_entropy(ro.W, om, 1.4) - O.total_entropy(Wo, om, 1.4)
    assert summ['deltaS'] == pytest.approx(dS, rel=1e-7, abs=1e-10)
    assert summ['stationarity_rel'] == pytest.approx(ro.final_residual, rel=1e-7)
    b = np.load(next((tmp_path / 'res').glob('*.npz')))
    for k in ("node_pos", "node_area", "conservatives", "primitives", "primitives_grad", "mach", "time", "mach_in",
              "aoa_in", "case", "mesh_path", "n_cells", "h", "flux", "reconstruction", "time_scheme"):
        assert k in b.files
    assert b['primitives_grad'].shape == (diamond02.n_cells, 4, 2)


def test_engineering_criterion_matches_oracle(diamond02, tmp_path):
    from eulersr_b200 import main as M
    from oracle import euler_oracle as O
    base = _cfg(stationarity_threshold=3e-4, stationarity_check_every=10, stationarity_patience=2)
    om = oracle_mesh(diamond02, np.float64)
    Wo, inl = O.initialize(diamond02.n_cells, base)
    ref = O.run(Wo, om, inl, dict(base))
    cd, cl = O.force_coefficients(ref.W, om, 1.0, 2.5 * math.sqrt(1.4), 1.0)
    cfg = dict(base, engineering_target_cd=cd * 1.002, engineering_target_cl=cl * 0.999,
               engineering_cd_tol=0.01, engineering_cl_tol=0.01, engineering_patience=2)
    ro = O.run(Wo, om, inl, dict(cfg))
    W0, inlet = M.initialize(diamond02, cfg)
    out = {'fig': tmp_path / 'f', 'res': tmp_path / 'r'}
    M.run(W0, diamond02, inlet, dict(cfg), out)
    summ = json.loads(next((tmp_path / 'r').glob('summary_*.json')).read_text())
    assert summ['engineering_converged'] == ro.eng_converged
    assert summ['engineering_stopping_step'] == ro.eng_stopping_step


def test_density_l2_rule_matches_oracle(diamond02):
    from eulersr_b200.solver import Solver, FlowCase
    from oracle import euler_oracle as O
    cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0, case='diamond', CFL=0.8, tf=3.0,
               stationarity_threshold=0.05, stationarity_check_every=20, stationarity_patience=1)
    om = oracle_mesh(diamond02, np.float64)
    W0, inl = O.initialize(diamond02.n_cells, cfg)
    ro = O.run(W0, om, inl, cfg, stop_rule='density_l2')
    s = Solver(diamond02, 1, precision='f64', stop_rule='density_l2', threshold=0.05, check_every=20)
    s.set_case(0, FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.8, tf=3.0))
    r = s.run()[0]
    assert bool(r['converged']) == ro.converged
    assert r['stopping_step'] == ro.stopping_step
    assert r['last_rel'] == pytest.approx(ro.last_rel, rel=1e-9)


def test_local_dt_matches_oracle(diamond02):
    from eulersr_b200.solver import Solver, FlowCase
    from oracle import euler_oracle as O
    om = oracle_mesh(diamond02, np.float64)
    W, inl = O.initialize(diamond02.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.0, aoa=2.0,
                                                   case='diamond'))
    for _ in range(25):
        W = O.time_step_srk2_local(W, om, 0.6, inl)
    s = Solver(diamond02, 1, precision='f64', dt_mode='local')
    s.set_case(0, FlowCase(mach=2.0, aoa_deg=2.0, cfl=0.6, tf=1.0, max_steps=10 ** 6))
    s.step(25)
    assert rel_err(s.get_state(0), W) <= 1e-12


def test_gradient_export_matches_oracle(diamond02):
    from eulersr_b200.solver import Solver, FlowCase
    from oracle import euler_oracle as O
    s = Solver(diamond02, 1, precision='f64')
    s.set_case(0, FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.6, tf=10.0))
    s.step(20)
    W = s.get_state(0)
    om = oracle_mesh(diamond02, np.float64)
    _, inl = O.initialize(diamond02.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0,
                                                  case='diamond'))
    WL = np.repeat(W[:, None], 3, axis=1)
    WR = O.bc_state(W[diamond02.neighbors], WL, om, inl)
    g = O.lsq_gradient(O.get_primitive(WL), O.get_primitive(WR), om)
    assert np.max(np.abs(s.gradients(0) - g)) <= 1e-10 * max(1.0, np.abs(g).max())


def test_subsonic_inlet_boundary(diamond02):
    """Marker 5 (helper.py:179-194): rho,u,v imposed from the mesh's subsonic
    inlet state, pressure from the cell."""
    from eulersr_b200.mesh import Mesh
    from eulersr_b200.solver import Solver, FlowCase, DeviceMesh
    from oracle import euler_oracle as O
    fm = diamond02.face_markers.copy()
    fm[fm == 3] = 5
    md = dict(diamond02.metadata, inlet_subsonic=[1.0, 0.6, 0.0, 1.0])
    m = Mesh.from_arrays(diamond02.points, diamond02.tris, diamond02.neighbors, diamond02.faces, fm,
                         diamond02.face_connectivity, md)
    om = oracle_mesh(m, np.float64)
    W, inl = O.initialize(m.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=0.5, aoa=0.0, case='diamond'))
    dt = O.get_dt(W, om, CFL=0.6)
    orig = O.bc_state
    O.bc_state = lambda WR, WL, mesh, inlet, wall_markers=None, inlet_subsonic=None: orig(
        WR, WL, mesh, inlet, wall_markers, [1.0, 0.6, 0.0, 1.0])
    try:
        for _ in range(15):
            W = O.time_step_srk2(W, om, dt, inl)
    finally:
        O.bc_state = orig
    s = Solver(DeviceMesh(m), 1, precision='f64')
    s.set_case(0, FlowCase(mach=0.5, aoa_deg=0.0, cfl=0.6, tf=10.0))
    s.step(15)
    assert rel_err(s.get_state(0), W) <= 1e-12


def test_worker_protocol(tmp_path, diamond02):
    mesh_path = tmp_path / 'diamond_h0.2.npz'
    diamond02.save(mesh_path)
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    base = [sys.executable, '-m', 'eulersr_b200.worker', '--case', 'diamond', '--mesh-path', str(mesh_path),
            '--mach', '2.5', '--aoa', '5', '--tf', '3.0', '--stationarity-threshold', '1e-3',
            '--scratch-dir', str(tmp_path / 'scratch'), '--precision', 'f64']
    r = subprocess.run(base + ['--stationarity-check-every', '10', '--stationarity-patience', '2', '--emit-summary'],
                       capture_output=True, text=True, env=env, cwd=str(ROOT), timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert 'Simulation terminée en' in r.stdout
    summ = json.loads(r.stdout.split('FVM_SUMMARY_JSON=')[1].splitlines()[0])
    assert summ['stationarity_patience'] == 2
    prim = np.tile([1.0, 2.5 * math.sqrt(1.4), 0.0, 1.0], (diamond02.n_cells, 1))
    np.save(tmp_path / 'init.npy', prim)
    r = subprocess.run(base + ['--init-field', str(tmp_path / 'init.npy'), '--probe-only'], capture_output=True,
                       text=True, env=env, cwd=str(ROOT), timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    probe = json.loads(r.stdout.split('FVM_PROBE_JSON=')[1].splitlines()[0])
    assert probe['residual'] > 0 and probe['dt'] > 0
    r = subprocess.run(base + ['--init-field', str(tmp_path / 'init.npy'), '--forces-only'], capture_output=True,
                       text=True, env=env, cwd=str(ROOT), timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    f = json.loads(r.stdout.split('FVM_FORCES_JSON=')[1].splitlines()[0])
    # uniform pressure p_inf on a closed body: zero net force
    assert abs(f['cd']) < 1e-9 and abs(f['cl']) < 1e-9


@pytest.fixture(scope="module")
def diamond_hr():
    from eulersr_b200.meshing import build_mesh
    return build_mesh('diamond', 0.025)


def test_diamond_shock_expansion_validation(diamond_hr):
    """The diamond checks at the reference's published validation point
    (diamond h=0.025, M=1.5, alpha=0; README.md:54-55 reports 1.8 % CD error
    and a 0.83 deg shock-angle error): converged CD vs shock-expansion theory,
    the leading-edge shock angle, and FP32 vs the FP64 build of the same
    kernels (CD within 1e-4 relative)."""
    from eulersr_b200.solver import Solver, FlowCase
    from eulersr_b200.postproc import diamond_theory, shock_angle_deg
    M = 1.5
    th = diamond_theory(M, 0.0, half_angle_deg=5.0)
    out = {}
    for prec in ('f64', 'f32'):
        s = Solver(diamond_hr, 1, precision=prec, threshold=1e-5, check_every=25)
        s.set_case(0, FlowCase(mach=M, aoa_deg=0.0, cfl=0.6, tf=30.0,
                               dtype=np.float64 if prec == 'f64' else np.float32))
        r = s.run()[0]
        out[prec] = (r, s.get_state(0))
    r64, W64 = out['f64']
    r32, W32 = out['f32']
    assert r64['converged'] and r32['converged']
    cd_err = abs(r64['cd'] - th.cd) / th.cd
    assert cd_err < 0.018, (r64['cd'], th.cd)
    beta = shock_angle_deg(diamond_hr, W64, le=(1.0, 2.0))
    assert abs(beta - th.beta_upper_deg) < 0.83, (beta, th.beta_upper_deg)
    assert abs(r32['cd'] - r64['cd']) <= 1e-4 * abs(r64['cd'])
    assert abs(r64['cl']) < 2e-3


def test_engineering_stop_rule_matches_oracle(diamond02):
    """ESR_STOP_ENGINEERING: the case ends when CD/CL stay within tolerance
    of their targets for `patience` checks; same step as the oracle."""
    from eulersr_b200.solver import Solver, FlowCase
    from oracle import euler_oracle as O
    base = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0, case='diamond', CFL=0.6, tf=3.0,
                stationarity_threshold=1e-12, stationarity_check_every=5, stationarity_patience=3)
    om = oracle_mesh(diamond02, np.float64)
    W0, inl = O.initialize(diamond02.n_cells, base)
    longrun = O.run(W0, om, inl, dict(base), max_steps=600)
    cd, cl = O.force_coefficients(longrun.W, om, 1.0, 2.5 * math.sqrt(1.4), 1.0)
    cfg = dict(base, engineering_target_cd=cd, engineering_target_cl=cl, engineering_cd_tol=0.005,
               engineering_cl_tol=0.005, engineering_patience=3)
    ro = O.run(W0, om, inl, dict(cfg), stop_rule='engineering')
    s = Solver(diamond02, 1, precision='f64', stop_rule='engineering', threshold=1e-12, check_every=5, patience=3)
    s.set_case(0, FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.6, tf=3.0, eng_target_cd=cd, eng_target_cl=cl,
                           eng_cd_tol=0.005, eng_cl_tol=0.005, eng_patience=3))
    r = s.run()[0]
    assert ro.converged and bool(r['converged'])
    assert r['stopping_step'] == ro.stopping_step == ro.eng_stopping_step
    assert rel_err(s.get_state(0), ro.W) <= 1e-10


def test_grid_batch_matches_single_runs(diamond02, tmp_path, capsys):
    """slurm/run_euler_grid.py on the batched solver: every case's summary,
    bundle and returned state equal those of main.run for the same case
    (two slots for five cases, so slots are refilled on the device)."""
    from eulersr_b200 import grid as G
    from eulersr_b200 import main as M
    cfg = _cfg(precision='f32', tf=1.0, stationarity_threshold=5e-4, stationarity_check_every=10)
    grid = [(1.5, -2.0), (1.5, 2.0), (2.5, 0.0), (0.9, 1.0), (3.0, 4.0)]
    recs = G.run_grid(cfg, diamond02, grid, slots=2, out_root=tmp_path / 'batch')
    capsys.readouterr()
    assert len(recs) == len(grid)
    for (mach, aoa), rec in zip(grid, recs):
        c = G.build_case_cfg(cfg, 'diamond', mach, aoa)
        W0, inlet = M.initialize(diamond02, c)
        dirs = {'fig': tmp_path / 'f', 'res': tmp_path / 'single' / f'{mach}_{aoa}'}
        W = M.run(W0, diamond02, inlet, c, dirs)
        assert np.array_equal(W, rec['W'])
        one = json.loads(next(dirs['res'].glob('summary_*.json')).read_text())
        tag = f"AOA{aoa:.2f}"
        batch = json.loads(next((tmp_path / 'batch').rglob(f'{tag}/summary_AOA{aoa:.2f}_M{mach:.2f}_*.json')).read_text())
        for k in ('cd', 'cl', 'converged', 'stopping_step', 'stationarity_rel', 'deltaS', 'mach', 'aoa', 'n_cells'):
            assert one[k] == batch[k], (mach, aoa, k, one[k], batch[k])
        b1 = np.load(next(dirs['res'].glob('*.npz')))
        b2 = np.load(next((tmp_path / 'batch').rglob(f'{tag}/AOA{aoa:.2f}_M{mach:.2f}_*.npz')))
        for k in ('conservatives', 'primitives', 'primitives_grad', 'mach', 'time'):
            assert np.array_equal(b1[k], b2[k]), k
