"""Drop-in for EulerSR's ``slurm/run_euler_grid.py``: a (Mach, AoA) grid on
one mesh, solved as one batch.

The reference loops over the grid and runs ``euler.main.run`` once per case
(``slurm/run_euler_grid.py:94-104``). Here every case of the grid goes into
one ``esr_batch_solve`` call: the slots of the mesh advance together, a slot
whose stop rule fires is refilled on the device with the next case, and the
outputs of each case (stdout line, bundle ``.npz`` with device LSQ gradients,
summary JSON) are written afterwards exactly as ``main.run`` writes them for
the same case. Each case's numbers are bitwise those of a single-case solve.

CLI: the reference's flags (``--case --mesh-path --mach --aoa --tf
--stationarity-threshold --verbose --dry-run``) plus ``--slots`` (cases in
flight, default min(#cases, 64)), ``--precision`` and ``--out-root``.
"""
from __future__ import annotations

import argparse
import copy
import itertools
import sys

import numpy as np

from . import main as euler_main
from .config import AOA_CASES_LC, KNOWN_CASES, KNOWN_CASES_LC, format_snapshot_name, load_mesh, setup_dirs
from .solver import FlowCase, Solver


def parse_range(spec: str):
    """slurm/run_euler_grid.py:24-31: 'start:stop:step', 'a,b,c' or one value."""
    if ":" in spec:
        start, stop, step = (float(x) for x in spec.split(":"))
        n = int(round((stop - start) / step))
        return [round(start + i * step, 10) for i in range(n + 1)]
    if "," in spec:
        return [round(float(x), 10) for x in spec.split(",") if x.strip()]
    return [round(float(spec), 10)]


def normalize_optional_value(argv, option_name: str):
    """slurm/run_euler_grid.py:34-47: '--aoa -5:5:1' -> '--aoa=-5:5:1' so a
    negative range is not read as a flag."""
    out, i = [], 0
    while i < len(argv):
        tok = argv[i]
        if tok == option_name and i + 1 < len(argv):
            val = argv[i + 1]
            if val.startswith("-") and not val.startswith("--"):
                out.append(f"{option_name}={val}")
                i += 2
                continue
        out.append(tok)
        i += 1
    return out


def build_case_cfg(base_cfg, case, mach, aoa):
    """slurm/run_euler_grid.py:50-56."""
    cfg = copy.deepcopy(base_cfg)
    cfg["case"] = case
    cfg["Mach"] = round(float(mach), 10)
    cfg["aoa"] = 0.0 if case == "bump" else round(float(aoa), 10)
    cfg["stationarity_threshold"] = float(cfg.get("stationarity_threshold", 1e-5))
    return cfg


def _flow_case(cfg, mesh, dtype):
    """The FlowCase main.run builds for ``cfg`` (transonic clamp applied to
    cfg first, euler/main.py:117-120)."""
    if 0.6 < cfg["Mach"] < 1.1 and cfg["CFL"] > 0.45:
        cfg["CFL"] = 0.45
    aoa = float(cfg.get("aoa", 0.0)) if str(cfg.get("case", "")).lower() in AOA_CASES_LC else 0.0
    tcd, tcl = cfg.get("engineering_target_cd"), cfg.get("engineering_target_cl")
    track = tcd is not None and tcl is not None
    patience = max(1, int(cfg.get("stationarity_patience", 1)))
    return FlowCase(mach=cfg["Mach"], aoa_deg=aoa, cfl=cfg["CFL"], tf=cfg["tf"], gamma=cfg["gamma"],
                    rho_inf=cfg["rho_inf"], p_inf=cfg["p_inf"],
                    l_ref=float(mesh.metadata.get("obstacle_length", 1.0) or 1.0), clamp=False, dtype=dtype,
                    eng_target_cd=tcd if track else None, eng_target_cl=tcl if track else None,
                    eng_cd_tol=float(cfg.get("engineering_cd_tol", 0.001)),
                    eng_cl_tol=float(cfg.get("engineering_cl_tol", 0.001)),
                    eng_patience=int(cfg.get("engineering_patience", patience)) if track else 0)


def run_grid(base_cfg, mesh, grid, slots=None, out_root=".", write=True):
    """Solve every (Mach, AoA) of ``grid`` on ``mesh`` in one batch and write
    each case's outputs. Returns one record per case (cfg, result, final
    residual, dS, final state)."""
    m = euler_main._as_mesh(mesh)
    case_name = base_cfg["case"]
    cfgs = [build_case_cfg(base_cfg, case_name, ma, a) for ma, a in grid]
    if not cfgs:
        return []
    prec = euler_main._precision(base_cfg)
    dtype = np.float64 if prec == "f64" else np.float32
    scheme = euler_main._TIME[str(base_cfg["time_scheme"]).upper()]
    thr = float(base_cfg.get("stationarity_threshold", 1e-5))
    every = int(base_cfg.get("stationarity_check_every"))
    patience = max(1, int(base_cfg.get("stationarity_patience", 1)))
    B = max(1, min(len(cfgs), int(slots) if slots else 64))
    s = Solver(euler_main._device_mesh(m), B, precision=prec, flux=str(base_cfg["flux"]),
               reconstruction=str(base_cfg["reconstruction"]), time_scheme=scheme, threshold=thr,
               check_every=every, patience=patience)
    cases = [_flow_case(c, m, dtype) for c in cfgs]
    res, states = s.batch_solve(cases, want_states=True)
    records = []
    # The batch returns each case's one-step residual probe of its final state
    # (euler/main.py:228-230). Entropy before and after and the LSQ gradients
    # of the bundle come from the device, B cases at a time: the freestream
    # start gives S0 as main.run computes it, the final state S and gradients.
    for c0 in range(0, len(cases), B):
        idx = list(range(c0, min(c0 + B, len(cases))))
        for j, i in enumerate(idx):
            s.set_case(j, cases[i])
        for j in range(len(idx), B):
            s.clear_slot(j)
        S0 = s.entropy()
        for j, i in enumerate(idx):
            s.set_state(j, states[i])
        S1 = s.entropy()
        for j, i in enumerate(idx):
            cfg, r = cfgs[i], res[i]
            W = states[i].astype(dtype)
            final_time = int(r["stopping_step"]) * float(r["dt"])
            rec = dict(cfg=cfg, result=r, final_residual=float(r["final_residual"]), dS=float(S1[j] - S0[j]), W=W)
            records.append(rec)
            if write:
                _write_case(rec, m, s, j, final_time, out_root, i + 1, len(cases))
    return records


def _write_case(rec, m, s, slot, final_time, out_root, idx, n):
    cfg, r = rec["cfg"], rec["result"]
    verbose = bool(cfg.get("verbose", True))
    exp = cfg["export"]
    if verbose:
        print("\n" + "=" * 78)
    print(f"Case {idx}/{n}: case={cfg['case']} Mach={cfg['Mach']} AoA={cfg.get('aoa', 0.0)}")
    out_dirs = setup_dirs(cfg, m, root=out_root)
    converged = bool(r["converged"])
    wall = float(r["solve_time_s"])
    res_ = rec["final_residual"]
    if verbose:
        print(f"Simulation terminée en {wall:.2f}s (converged={converged}, t={final_time:.4f}s)")
        print(f"Résidu final : {res_:.6e}")
    else:
        print(f"Simulation terminée en {wall:.2f}s (converged={converged}, t={final_time:.4f}s, résidu={res_:.2e})")
    if exp.get("results") or exp.get("figures") or exp.get("bundle", True):
        euler_main.export_snapshot(rec["W"], m, s, final_time, cfg, out_dirs, slot=slot)
    if exp.get("graph"):
        from pathlib import Path
        m.save(Path(out_dirs["res"]) / "graph.npz", W_snapshots={round(final_time, 6): rec["W"]})
    if str(cfg["case"]).lower() in KNOWN_CASES_LC and exp.get("summary", True):
        tcd, tcl = cfg.get("engineering_target_cd"), cfg.get("engineering_target_cl")
        track = tcd is not None and tcl is not None
        summary = euler_main.build_run_summary(
            cfg, m, float(r["cd"]), float(r["cl"]), rec["dS"], wall, res_, converged, int(r["stopping_step"]),
            0.0, wall, max(1, int(cfg.get("stationarity_patience", 1))),
            bool(r["eng_converged"]) if track else None, int(r["eng_stopping_step"]) if track else None,
            tcd if track else None, tcl if track else None)
        euler_main.export_run_summary(out_dirs, summary, format_snapshot_name(cfg, final_time), verbose=verbose)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=KNOWN_CASES, required=True)
    ap.add_argument("--mesh-path", required=True)
    ap.add_argument("--mach", default="0.7:1.5:0.1")
    ap.add_argument("--aoa", default="0:0:1")
    ap.add_argument("--tf", type=float, default=None)
    ap.add_argument("--stationarity-threshold", type=float, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--dry-run", action="store_true")
    ap.add_argument("--slots", type=int, default=None)
    ap.add_argument("--precision", choices=("f32", "f64"), default=None)
    ap.add_argument("--out-root", default=".")
    argv = sys.argv[1:] if argv is None else list(argv)
    a = ap.parse_args(normalize_optional_value(argv, "--aoa"))
    base = copy.deepcopy(euler_main.CFG)
    base["case"] = a.case
    base["mesh_path"] = a.mesh_path
    base["verbose"] = bool(a.verbose)
    if a.tf is not None:
        base["tf"] = float(a.tf)
    if a.stationarity_threshold is not None:
        base["stationarity_threshold"] = float(a.stationarity_threshold)
    if a.precision:
        base["precision"] = a.precision
    machs = parse_range(a.mach)
    aoas = [0.0] if a.case == "bump" else parse_range(a.aoa)
    grid = list(itertools.product(machs, aoas))
    mesh = load_mesh(base)
    print(f"Loaded mesh once: {mesh.metadata.get('name', 'unknown')}")
    print(f"Cases to run: {len(grid)}")
    if a.dry_run:
        for ma, al in grid:
            print(f"case={a.case} Mach={ma} AoA={al}")
        return 0
    run_grid(base, mesh, grid, slots=a.slots, out_root=a.out_root)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
