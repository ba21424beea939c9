"""Drop-in for EulerSR's ``euler/main.py``: ``initialize`` and ``run``.

``run`` keeps the reference's behaviour and side effects: scheme selection
(unknown time scheme -> KeyError, unknown flux/reconstruction -> ValueError),
the transonic CFL clamp, dt computed once from the initial field,
N = int(tf/dt)+1, the stationarity rule with patience, the engineering
criterion, the final one-step residual probe, the stdout line that
``eval/live_fvm.py`` parses, the bundle ``.npz`` and the summary JSON
(``euler/main.py:43-270``, ``euler/utils.py:21-192``). Every solve step runs
in the CUDA kernels of ``libeulersr.so``.

Precision: ``cfg['precision']`` ('f32'/'f64') or, like JAX, float64 when the
environment sets ``JAX_ENABLE_X64=true`` (the reference's dataset and eval
runs do), float32 otherwise.
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

from .config import AOA_CASES_LC, KNOWN_CASES_LC, build_config_from_cli, format_snapshot_name, \
    load_default_config, load_mesh, setup_dirs
from .mesh import Mesh
from .solver import DeviceMesh, FlowCase, Solver, freestream

CFG = load_default_config()

_TIME = {"EE": "EE", "RK2": "RK2", "SRK2": "SRK2", "SSP_RK2": "SRK2"}
_SOLVERS: dict = {}


def _precision(cfg) -> str:
    p = cfg.get("precision")
    if p:
        return str(p).lower()
    return "f64" if os.environ.get("JAX_ENABLE_X64", "").lower() in ("1", "true", "yes") else "f32"


def _as_mesh(mesh) -> Mesh:
    """Accept the reference's Mesh object (JAX or NumPy arrays) or ours."""
    if isinstance(mesh, Mesh):
        return mesh
    m = Mesh.from_arrays(np.asarray(mesh.points), np.asarray(mesh.tris), np.asarray(mesh.neighbors),
                         np.asarray(mesh.faces), np.asarray(mesh.face_markers),
                         np.asarray(mesh.face_connectivity), dict(getattr(mesh, "metadata", {}) or {}))
    return m


def _device_mesh(mesh: Mesh) -> DeviceMesh:
    dm = getattr(mesh, "_esr_device_mesh", None)
    if dm is None:
        dm = DeviceMesh(mesh)
        mesh._esr_device_mesh = dm
    return dm


def _solver(mesh: Mesh, prec, flux, recon, scheme, thr, every, patience) -> Solver:
    """One cached solver per mesh and scheme: a grid of cases reuses its
    device buffers and captured graphs."""
    key = (id(mesh), prec, flux.lower(), recon.lower(), scheme, float(thr), int(every), int(patience))
    s = _SOLVERS.get(key)
    if s is None:
        s = Solver(_device_mesh(mesh), 1, precision=prec, flux=flux, reconstruction=recon, time_scheme=scheme,
                   threshold=thr, check_every=every, patience=patience)
        _SOLVERS[key] = s
    return s


def initialize(mesh, cfg):
    """euler/main.py:28-41: freestream W (N,4) and the conserved inlet state."""
    prec = _precision(cfg)
    dtype = np.float64 if prec == "f64" else np.float32
    aoa = float(cfg.get("aoa", 0.0)) if str(cfg.get("case", "")).lower() in AOA_CASES_LC else 0.0
    inlet = freestream(cfg["Mach"], aoa, cfg["gamma"], cfg["rho_inf"], cfg["p_inf"], dtype)
    n = int(np.asarray(mesh.area).shape[0])
    W = np.tile(inlet[None, :], (n, 1))
    return W, inlet


def _primitive(W, gamma):
    rho = W[:, 0]
    u = W[:, 1] / rho
    v = W[:, 2] / rho
    p = (W[:, 3] - 0.5 * rho * (u ** 2 + v ** 2)) * (gamma - 1)
    return np.stack([rho, u, v, p], -1)


def run(W, mesh, inlet, cfg, out_dirs):
    """euler/main.py:43-270 on the GPU."""
    verbose = bool(cfg.get("verbose", True))
    scheme = _TIME[str(cfg["time_scheme"]).upper()]          # KeyError like the reference
    flux = str(cfg["flux"])
    recon = str(cfg["reconstruction"])
    exp = cfg["export"]
    thr = float(cfg.get("stationarity_threshold"))
    every = int(cfg.get("stationarity_check_every"))
    patience = max(1, int(cfg.get("stationarity_patience", 1)))
    target_cd, target_cl = cfg.get("engineering_target_cd"), cfg.get("engineering_target_cl")
    track = target_cd is not None and target_cl is not None
    m = _as_mesh(mesh)
    if track:
        if m.metadata.get("obstacle_length") is None:
            raise ValueError("engineering_target_cd/cl given but mesh.metadata has no 'obstacle_length'")
        if not np.any(m.face_markers == m.force_marker()):
            raise ValueError(f"no wall face (force_marker={m.force_marker()}) in this mesh")
    if 0.6 < cfg["Mach"] < 1.1 and cfg["CFL"] > 0.45:
        if verbose:
            print(f"Attention : régime transsonique avec CFL={cfg['CFL']} potentiellement instable. CFL réduite à 0.45")
        cfg["CFL"] = 0.45
    prec = _precision(cfg)
    dtype = np.float64 if prec == "f64" else np.float32
    W = np.asarray(W)
    W_initial = W
    L_ref = float(m.metadata.get("obstacle_length", 1.0) or 1.0)
    aoa = float(cfg.get("aoa", 0.0)) if str(cfg.get("case", "")).lower() in AOA_CASES_LC else 0.0

    t0 = time.perf_counter()
    s = _solver(m, prec, flux, recon, scheme, thr, every, patience)
    case = FlowCase(mach=cfg["Mach"], aoa_deg=aoa, cfl=cfg["CFL"], tf=cfg["tf"], gamma=cfg["gamma"],
                    rho_inf=cfg["rho_inf"], p_inf=cfg["p_inf"], l_ref=L_ref, clamp=False, dtype=dtype,
                    eng_target_cd=target_cd if track else None, eng_target_cl=target_cl if track else None,
                    eng_cd_tol=float(cfg.get("engineering_cd_tol", 0.001)),
                    eng_cl_tol=float(cfg.get("engineering_cl_tol", 0.001)),
                    eng_patience=int(cfg.get("engineering_patience", patience)) if track else 0)
    s.set_case(0, case, W_init=np.asarray(W, dtype=np.float64))
    dt = float(s.dt()[0])
    S0 = float(s.entropy()[0])
    compile_time_s = time.perf_counter() - t0
    if verbose:
        N = int(cfg["tf"] / dtype(dt)) + 1
        print(f"    dt={dt:.2e}, Nt={N}, n_snaps={max(1, int(exp.get('n_snaps', 1)))}")
        print("\nRésolution numérique en cours...")
    t1 = time.perf_counter()
    r = s.run()[0]
    solve_time_s = time.perf_counter() - t1
    converged = bool(r["converged"])
    stopping_step = int(r["stopping_step"])
    final_residual = float(s.residual_probe()[0])
    W = s.get_state(0).astype(dtype)
    wall_time_s = compile_time_s + solve_time_s
    final_time = stopping_step * dt
    name = format_snapshot_name(cfg, final_time)
    if verbose:
        print("\n" + "-" * 78)
        print(f"Simulation terminée en {wall_time_s:.2f}s (converged={converged}, t={final_time:.4f}s)")
        print(f"Résidu final : {final_residual:.6e}")
    else:
        print(f"Simulation terminée en {wall_time_s:.2f}s (converged={converged}, t={final_time:.4f}s, "
              f"résidu={final_residual:.2e})")
    if exp.get("results") or exp.get("figures") or exp.get("bundle", True):
        export_snapshot(W, m, s, final_time, cfg, out_dirs)
    if exp.get("graph"):
        m.save(Path(out_dirs["res"]) / "graph.npz", W_snapshots={round(final_time, 6): W}, inlet_state=inlet)
    if str(cfg["case"]).lower() in KNOWN_CASES_LC and exp.get("summary", True):
        cd, cl = float(r["cd"]), float(r["cl"])
        dS = float(s.entropy()[0]) - S0
        if verbose:
            print(f"C_D = {cd:.6f}, C_L = {cl:.6f}, ΔS = {dS:.6e}")
        summary = build_run_summary(cfg, m, cd, cl, dS, wall_time_s, final_residual, converged, stopping_step,
                                    compile_time_s, solve_time_s, patience,
                                    bool(r["eng_converged"]) if track else None,
                                    int(r["eng_stopping_step"]) if track else None,
                                    target_cd if track else None, target_cl if track else None)
        export_run_summary(out_dirs, summary, name, verbose=verbose)
    return W


def export_snapshot(W, mesh: Mesh, s: Solver, t, cfg, out_dirs, slot: int = 0):
    """euler/utils.py:21-69: .npy state and the bundle .npz (primitives, LSQ
    primitive gradients of solver slot ``slot`` from the device, Mach)."""
    exp, gamma = cfg["export"], cfg["gamma"]
    name = format_snapshot_name(cfg, t)
    res = Path(out_dirs["res"])
    res.mkdir(parents=True, exist_ok=True)
    if exp.get("results"):
        np.save(res / f"{name}.npy", np.asarray(W))
    if exp.get("bundle", True):
        prims = _primitive(np.asarray(W, np.float64), gamma)
        grad = s.gradients(slot)
        mach = np.sqrt(prims[:, 1] ** 2 + prims[:, 2] ** 2) / np.sqrt(gamma * prims[:, 3] / prims[:, 0])
        path = res / f"{name}.npz"
        if cfg.get("verbose", True):
            print(f"Bundle export : {path}")
        np.savez_compressed(
            path, node_pos=mesh.barycenter.astype(np.float32), node_area=mesh.area.astype(np.float32),
            conservatives=np.asarray(W, np.float32), primitives=prims.astype(np.float32),
            primitives_grad=grad.astype(np.float32), mach=mach.astype(np.float32),
            time=np.asarray([float(t)], np.float32), mach_in=np.asarray([float(cfg["Mach"])], np.float32),
            aoa_in=np.asarray([float(cfg.get("aoa", 0.0))], np.float32), case=np.asarray([str(cfg.get("case", ""))]),
            mesh_path=np.asarray([str(cfg.get("mesh_path", ""))]), n_cells=np.asarray([mesh.n_cells]),
            h=np.asarray([float(mesh.metadata.get("h", float("nan")))]), flux=np.asarray([str(cfg.get("flux", ""))]),
            reconstruction=np.asarray([str(cfg.get("reconstruction", ""))]),
            time_scheme=np.asarray([str(cfg.get("time_scheme", ""))]))


def build_run_summary(cfg, mesh, cd, cl, delta_s, wall_time_s, stationarity_rel=None, converged=None,
                      stopping_step=None, compile_time_s=None, solve_time_s=None, stationarity_patience=None,
                      engineering_converged=None, engineering_stopping_step=None, engineering_target_cd=None,
                      engineering_target_cl=None) -> dict:
    """euler/utils.py:147-182 (same keys)."""
    f = lambda v: float(v) if v is not None else None
    i = lambda v: int(v) if v is not None else None
    return {
        "case": cfg["case"], "h": mesh.metadata.get("h"), "n_cells": int(mesh.n_cells),
        "cd": f(cd), "cl": f(cl), "deltaS": f(delta_s), "stationarity_rel": f(stationarity_rel),
        "converged": bool(converged) if converged is not None else None, "stopping_step": i(stopping_step),
        "stationarity_threshold": f(cfg.get("stationarity_threshold")),
        "stationarity_check_every": i(cfg.get("stationarity_check_every")),
        "stationarity_patience": i(stationarity_patience), "wall_time_s": float(wall_time_s),
        "compile_time_s": f(compile_time_s), "solve_time_s": f(solve_time_s),
        "engineering_converged": bool(engineering_converged) if engineering_converged is not None else None,
        "engineering_stopping_step": i(engineering_stopping_step),
        "engineering_target_cd": f(engineering_target_cd), "engineering_target_cl": f(engineering_target_cl),
        "time_scheme": cfg["time_scheme"], "flux": cfg["flux"], "reconstruction": cfg["reconstruction"],
        "mach": cfg["Mach"], "mesh_path": cfg["mesh_path"], "aoa": float(cfg.get("aoa", 0.0)),
    }


def export_run_summary(out_dirs, summary, snapshot_name, verbose=True):
    res = Path(out_dirs["res"])
    res.mkdir(parents=True, exist_ok=True)
    path = res / f"summary_{snapshot_name}.json"
    path.write_text(json.dumps(summary, indent=2))
    if verbose:
        print(f"Summary written : {path}")


if __name__ == "__main__":
    CFG = build_config_from_cli(CFG)
    mesh = load_mesh(CFG)
    out_dirs = setup_dirs(CFG, mesh)
    W0, inlet0 = initialize(mesh, CFG)
    run(W0, mesh, inlet0, CFG, out_dirs)
