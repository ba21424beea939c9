"""Command-line solve with the protocol of EulerSR's eval worker.

Same flags and stdout lines as ``eval/_fvm_solve_worker.py:31-155``: the
"Simulation terminée en Xs" line, ``FVM_SUMMARY_JSON=`` with
``--emit-summary``, ``FVM_PROBE_JSON=`` with ``--probe-only`` (one-step
relative residual and dt of a given primitive field) and ``FVM_FORCES_JSON=``
with ``--forces-only``. ``eval/live_fvm.py`` can call it instead of the JAX
worker (``python -m eulersr_b200.worker ...``); the solve runs on the GPU in
this process.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument('--case', required=True)
    ap.add_argument('--mesh-path', required=True)
    ap.add_argument('--mach', type=float, required=True)
    ap.add_argument('--aoa', type=float, required=True)
    ap.add_argument('--tf', type=float, required=True)
    ap.add_argument('--stationarity-threshold', type=float, required=True)
    ap.add_argument('--scratch-dir', required=True)
    ap.add_argument('--stationarity-check-every', type=int, default=None)
    ap.add_argument('--stationarity-patience', type=int, default=1)
    ap.add_argument('--target-cd', type=float, default=None)
    ap.add_argument('--target-cl', type=float, default=None)
    ap.add_argument('--cd-tol', type=float, default=0.001)
    ap.add_argument('--cl-tol', type=float, default=0.001)
    ap.add_argument('--engineering-patience', type=int, default=None)
    ap.add_argument('--init-field', default=None, help='(N,4) primitive field (.npy) for a warm start')
    ap.add_argument('--emit-summary', action='store_true')
    ap.add_argument('--probe-only', action='store_true')
    ap.add_argument('--forces-only', action='store_true')
    ap.add_argument('--precision', choices=('f32', 'f64'), default=None)
    args = ap.parse_args(argv)

    from . import main as M
    from .config import load_default_config, load_mesh
    from .solver import FlowCase

    cfg = load_default_config()
    cfg.update(case=args.case, Mach=args.mach, aoa=args.aoa, mesh_path=args.mesh_path, tf=args.tf,
               stationarity_threshold=args.stationarity_threshold, verbose=False)
    if args.precision:
        cfg['precision'] = args.precision
    if args.stationarity_check_every is not None:
        cfg['stationarity_check_every'] = args.stationarity_check_every
    cfg['stationarity_patience'] = max(1, int(args.stationarity_patience))
    if args.target_cd is not None and args.target_cl is not None:
        cfg['engineering_target_cd'] = float(args.target_cd)
        cfg['engineering_target_cl'] = float(args.target_cl)
        cfg['engineering_cd_tol'] = float(args.cd_tol)
        cfg['engineering_cl_tol'] = float(args.cl_tol)
        cfg['engineering_patience'] = (int(args.engineering_patience) if args.engineering_patience is not None
                                       else cfg['stationarity_patience'])
    cfg['export'] = dict(results=False, figures=[], graph=False, summary=bool(args.emit_summary), bundle=False,
                         n_snaps=1)
    mesh = load_mesh(cfg)
    scratch = Path(args.scratch_dir)
    out_dirs = {'fig': scratch / 'fig', 'res': scratch / 'res'}
    for d in out_dirs.values():
        d.mkdir(parents=True, exist_ok=True)

    W, inlet = M.initialize(mesh, cfg)
    if args.init_field:
        prim = np.load(args.init_field)
        if prim.shape != (mesh.n_cells, 4):
            raise ValueError(f"--init-field has shape {prim.shape}, expected ({mesh.n_cells}, 4) for this mesh.")
        rho, u, v, p = (prim[:, i].astype(np.float64) for i in range(4))
        W = np.stack([rho, rho * u, rho * v, p / (cfg['gamma'] - 1) + 0.5 * rho * (u ** 2 + v ** 2)], -1)

    if args.forces_only or args.probe_only:
        if not args.init_field:
            raise SystemExit('--forces-only / --probe-only need --init-field.')
        if 0.6 < cfg['Mach'] < 1.1 and cfg['CFL'] > 0.45:
            cfg['CFL'] = 0.45
        L_ref = mesh.metadata.get('obstacle_length')
        if args.forces_only and L_ref is None:
            raise SystemExit(f"mesh.metadata has no 'obstacle_length' (case='{args.case}').")
        prec = M._precision(cfg)
        s = M._solver(mesh, prec, cfg['flux'], cfg['reconstruction'], M._TIME[str(cfg['time_scheme']).upper()],
                      1e-30, 1, 1)
        s.set_case(0, FlowCase(mach=cfg['Mach'], aoa_deg=cfg['aoa'], cfl=cfg['CFL'], tf=cfg['tf'],
                               l_ref=float(L_ref or 1.0), clamp=False,
                               dtype=np.float64 if prec == 'f64' else np.float32), W_init=W)
        if args.forces_only:
            cd, cl = s.forces()
            print('FVM_FORCES_JSON=' + json.dumps({'cd': float(cd[0]), 'cl': float(cl[0])}))
        else:
            rel = float(s.residual_probe()[0])
            print('FVM_PROBE_JSON=' + json.dumps({'residual': rel, 'dt': float(s.dt()[0])}))
        return 0

    if args.emit_summary:
        for stale in out_dirs['res'].glob('summary_*.json'):
            stale.unlink()
    M.run(W, mesh, inlet, cfg, out_dirs)
    if args.emit_summary:
        found = sorted(out_dirs['res'].glob('summary_*.json'))
        if not found:
            raise RuntimeError(f"--emit-summary requested but no summary was written (case='{args.case}').")
        print('FVM_SUMMARY_JSON=' + json.dumps(json.loads(found[-1].read_text())))
    return 0


if __name__ == '__main__':
    sys.exit(main())
