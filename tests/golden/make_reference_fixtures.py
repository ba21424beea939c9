"""Golden vectors from EulerSR's own NumPy utilities, for the CPU tests.

The reference's solver needs JAX, which is not installed, but three of its
host utilities import with NumPy and SciPy alone; this script runs them on
seeded inputs and stores inputs and outputs in ``reference_utils.npz``:

* ``utils/metrics.py:9-14`` idw_weights (p = 2 inverse-distance weights);
* ``utils/aero.py:154-177`` wall_features (wall distance and normal);
* ``utils/aero.py:28-72,85-110`` build_wall_cache + aero_coeffs (CL, CD);
* ``euler/graph.py:5-108`` export_graph on the golden diamond mesh with one
  seeded snapshot, written by the reference itself as ``reference_graph.npz``;
* ``euler/config.py:24-62,82-103`` the default configuration, the command
  line's configurations for a few argument lists and the output naming (h
  tag, condition tag, snapshot name) into ``reference_config.json``;
* ``euler/utils.py:147-191`` build_run_summary and export_run_summary (the
  module imports matplotlib, which is not installed, so these two functions
  are taken from its source alone and run with NumPy), their summaries and
  the written file's name and text into ``reference_summary.json``;
* the reference's own solver source (``reference_solver_run.py``: mesh
  geometry, initialize, dt, boundary states, LSQ gradient, limiter, MUSCL,
  HLLC, sponge, residual, SRK2) with NumPy standing in for jax.numpy: 20 SRK2
  steps of the supersonic diamond (M 2.5, alpha 5) and the transonic NACA0012
  (M 0.8, alpha 1.25) golden meshes in float32 and float64, with their dt,
  CD, CL and entropy created, plus 10 steps of the diamond with the Rusanov
  flux, constant reconstruction, explicit Euler and RK2, into
  ``reference_solver.npz``; the same 20 steps on the HR diamond of the
  single-case HR workload (h = 0.025 by the package's mesher, 19,384 cells,
  M 2.0, alpha 0) in float32 and float64 into ``reference_solver_hr.npz``
  (``--hr-only`` writes just that one); and ``euler/main.py:43-270`` itself (the
  stepping loop with the stationarity rule, the engineering criterion and
  the stop bookkeeping, exports off) on three configurations, final states
  and stop records into ``reference_runs.npz``;
* ``euler/postproc/theory_validation_diamond.py:44-175`` the shock-expansion
  panel states of the diamond (same treatment: the gas-dynamics functions
  taken from the source, run with NumPy and SciPy) for a set of Mach numbers
  and incidences, and its campaign helpers (``:237-342,609-621``: plateau
  values, shock-angle measurement, log-log order fit) and the mesh-convergence
  helpers (``mesh_convergence_diamond.py:106-161``: profile error, GCI) on
  seeded inputs, into ``reference_theory.json`` (the helpers' array inputs
  in ``reference_theory_inputs.npz``).

Run from the repository root with the reference checkout as the argument:

    python tests/golden/make_reference_fixtures.py <path of the EulerSR checkout>
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def main(ref_root: str) -> Path:
    sys.path.insert(0, str(ROOT))
    from eulersr_b200.mesh import Mesh
    sys.dont_write_bytecode = True                     # nothing is written into the reference checkout
    sys.path.insert(0, str(Path(ref_root)))
    from utils.aero import aero_coeffs, build_wall_cache, wall_features
    from utils.metrics import idw_weights
    sys.path.insert(0, str(Path(ref_root) / "euler"))
    from graph import export_graph
    import config as ref_config

    mesh = Mesh.load(HERE / "diamond_h0.2.npz")
    rng = np.random.default_rng(11)
    dist = rng.uniform(1e-4, 0.5, (500, 6))
    dist[:5, 0] = 0.0                                  # coincident points: the eps term decides
    w = idw_weights(dist)
    query = np.concatenate([mesh.barycenter, rng.uniform([0.5, 1.5], [2.5, 2.5], (300, 2))])
    wd, wn = wall_features(mesh, query)
    n = mesh.n_cells
    prim = np.stack([rng.uniform(0.5, 2.0, n), rng.uniform(0.5, 3.0, n), rng.uniform(-0.5, 0.5, n),
                     rng.uniform(0.5, 3.0, n)], 1)
    mach = 2.0
    ac = aero_coeffs(prim, build_wall_cache(mesh), mach)
    snap = rng.standard_normal((n, 4))
    export_graph(mesh, {0.5: snap, 1.25: 2 * snap}, [1.0, 2.0, 0.1, 4.5], str(HERE / "reference_graph.npz"))
    names = []
    base = ref_config.load_default_config()
    for case, m_c, a_c, t, h in (("diamond", 2.5, 5.0, 1.234, 0.025), ("naca0012", 0.8, -2.5, 10.0, 0.1),
                                 ("bump", 1.4, 3.0, 0.5, 0.05), ("NACA2412", 3.0, 0.0, 123.456, None),
                                 ("rae2822", 0.75, 2.31, 7.0, 0.0125)):
        cfg = dict(base, case=case, Mach=m_c, aoa=a_c)
        mesh_h = type("M", (), {"metadata": {} if h is None else {"h": h}})()
        names.append(dict(case=case, Mach=m_c, aoa=a_c, t=t, h=h, h_tag=ref_config.format_h(mesh_h),
                          condition=ref_config.format_condition_tag(cfg),
                          snapshot=ref_config.format_snapshot_name(cfg, t)))
    cli = []
    saved = sys.argv
    for argv in (["--case", "naca0012", "--mach", "0.8", "--aoa", "-2.5"],
                 ["--time-scheme", "SSP_RK2", "--reconstruction", "muscl", "--quiet"],
                 ["--flux", "Rusanov", "--reconstruction", "constant", "--time-scheme", "EE",
                  "--stationarity-threshold", "1e-5", "--stationarity-check-every", "0",
                  "--stationarity-patience", "3", "--mesh-path", "m.npy"]):
        sys.argv = ["main.py", *argv]
        cli.append({"argv": argv, "cfg": ref_config.build_config_from_cli(base)})
    sys.argv = saved
    (HERE / "reference_config.json").write_text(json.dumps({"default": base, "names": names, "cli": cli},
                                                           indent=1, sort_keys=True) + "\n")
    sys.path.insert(0, str(HERE))
    import reference_solver_run as RS
    solver = {}
    for tag, name, m_s, a_s in (("diamond", "diamond_h0.2", 2.5, 5.0), ("naca", "naca0012_h0.2", 0.8, 1.25)):
        m = Mesh.load(HERE / f"{name}.npz")
        for dname, dtp in (("f32", np.float32), ("f64", np.float64)):
            W, dt_, cd, cl, ds = RS.run(ref_root, m, m_s, a_s, 20, dtp, ref_config._AOA_CASES_LC, diagnostics=True)
            solver[f"{tag}_{dname}_W20"] = W
            solver[f"{tag}_{dname}_dt"] = np.asarray(dt_, dtype=dtp)
            solver[f"{tag}_{dname}_cd_cl_dS"] = np.array([cd, cl, ds])
    dmesh = Mesh.load(HERE / "diamond_h0.2.npz")
    for flux, rec, sch in (("Rusanov", "MUSCL", "SRK2"), ("HLLC", "constant", "SRK2"), ("HLLC", "MUSCL", "EE"),
                           ("HLLC", "MUSCL", "RK2")):
        for dname, dtp in (("f32", np.float32), ("f64", np.float64)):
            W, _ = RS.run(ref_root, dmesh, 2.5, 5.0, 10, dtp, ref_config._AOA_CASES_LC, flux=flux,
                          reconstruction=rec, scheme=sch)
            solver[f"variant_{flux}_{rec}_{sch}_{dname}_W10"] = W
    np.savez_compressed(HERE / "reference_solver.npz", **solver)
    runs, cfgs = {}, {}
    base = ref_config.load_default_config()
    eng = dict(engineering_target_cd=0.1235, engineering_target_cl=0.0635, engineering_cd_tol=0.3,
               engineering_cl_tol=0.3, engineering_patience=2)
    for tag, name, extra, precs in (
            ("diamond", "diamond_h0.2", dict(case="diamond", Mach=2.5, aoa=5.0, tf=0.5, stationarity_threshold=2e-3,
                                             stationarity_check_every=10, stationarity_patience=2), ("f32", "f64")),
            ("naca_eng", "naca0012_h0.2", dict(case="naca0012", Mach=0.8, aoa=1.25, tf=0.3, stationarity_threshold=2e-4,
                                               stationarity_check_every=7, stationarity_patience=3, **eng), ("f32", "f64")),
            ("naca_cap", "naca0012_h0.2", dict(case="naca0012", Mach=0.8, aoa=1.25, tf=0.3, stationarity_threshold=5e-5,
                                               stationarity_check_every=7, stationarity_patience=3, **eng), ("f64",))):
        m = Mesh.load(HERE / f"{name}.npz")
        cfg = dict(base, **extra)
        cfgs[tag] = {k: v for k, v in cfg.items() if k != "export"}
        for prec in precs:
            W, carry = RS.run_main(ref_root, m, dict(cfg), np.float32 if prec == "f32" else np.float64,
                                   ref_config._AOA_CASES_LC, ref_config._KNOWN_CASES_LC, ref_config.format_snapshot_name)
            runs[f"{tag}_{prec}_W"] = W
            runs[f"{tag}_{prec}_stop"] = np.array([bool(carry[4]), int(carry[6]), bool(carry[9]), int(carry[12])],
                                                  dtype=np.int64)
    runs["cfgs_json"] = np.array(json.dumps(cfgs, sort_keys=True))
    np.savez_compressed(HERE / "reference_runs.npz", **runs)
    theory = _theory(Path(ref_root) / "euler" / "postproc" / "theory_validation_diamond.py")
    (HERE / "reference_theory.json").write_text(json.dumps(theory, indent=1, sort_keys=True) + "\n")
    summaries = _summaries(Path(ref_root) / "euler" / "utils.py")
    (HERE / "reference_summary.json").write_text(json.dumps(summaries, indent=1, sort_keys=True) + "\n")
    out = HERE / "reference_utils.npz"
    np.savez_compressed(out, graph_snapshot=snap, idw_dist=dist, idw_w=w, wall_query=query, wall_dist=wd, wall_normal=wn,
                        aero_prim=prim, aero_mach=np.float64(mach), aero_cl=np.float64(ac["CL"]),
                        aero_cd=np.float64(ac["CD"]))
    return out


def _theory(src: Path) -> list:
    """Panel states (Mach, pressure ratio to freestream, Cp, shock angle,
    attached) of the reference's diamond_panels for several (M, alpha)."""
    import ast
    import dataclasses
    from scipy.optimize import brentq
    names = {"prandtl_meyer", "inverse_prandtl_meyer", "_theta_of_beta", "theta_max", "oblique_shock_beta",
             "PanelState", "_apply_deflection", "diamond_panels", "all_attached", "_panel_of", "_plateau_value",
             "_panel_masks", "_measure_shock_angle", "fit_order", "richardson_gci", "_relative_profile_error",
             "SHOCK_WINDOW_X", "SHOCK_WINDOW_Y_FACTOR", "SHOCK_TOP_PCT", "H_GCI"}

    def wanted(n):
        if isinstance(n, (ast.FunctionDef, ast.ClassDef)):
            return n.name in names
        return (isinstance(n, ast.Assign) and len(n.targets) == 1 and isinstance(n.targets[0], ast.Name)
                and n.targets[0].id in names)
    tree = ast.parse(src.read_text())
    conv = ast.parse((src.parent / "mesh_convergence_diamond.py").read_text())
    keep = [n for n in conv.body if wanted(n)] + [n for n in tree.body if wanted(n)]
    import types
    mod = types.ModuleType("reference_theory")     # dataclass() looks its module up in sys.modules
    mod.__dict__.update(np=np, brentq=brentq, dataclass=dataclasses.dataclass, GAMMA=1.4)
    sys.modules[mod.__name__] = mod
    try:
        exec(compile(ast.Module(body=keep, type_ignores=[]), str(src), "exec"), mod.__dict__)
    finally:
        del sys.modules[mod.__name__]
    ns = mod.__dict__
    out = {"panels": [], "helpers": {}}
    rng = np.random.default_rng(17)
    # plateau values on a synthetic two-sided wall profile around (1.5, 2.0)
    x = np.sort(rng.uniform(1.0, 2.0, 80))
    y = 2.0 + np.where(np.arange(80) % 2 == 0, 1.0, -1.0) * 0.05 * (1 - np.abs(x - 1.5) / 0.5)
    prof = {"x": x, "y": y, "p": rng.uniform(0.5, 2.0, 80), "mach": rng.uniform(1.0, 3.0, 80)}
    masks = ns["_panel_masks"](prof, 1.5, 2.0)
    arrays = {f"profile_{k}": v for k, v in prof.items()}
    out["helpers"]["plateau_p"] = ns["_plateau_value"](prof, masks, "p", lambda p: (p - 1.0) / 2.8)
    out["helpers"]["plateau_mach"] = ns["_plateau_value"](prof, masks, "mach", lambda m: m)
    # shock angle from a gradient ridge through the leading edge at 40 degrees, jittered
    pos = np.column_stack([rng.uniform(0.6, 1.5, 2000), rng.uniform(1.7, 2.3, 2000)])
    dist = np.abs(np.sin(np.radians(40.0)) * (pos[:, 0] - 1.0) - np.cos(np.radians(40.0)) * (pos[:, 1] - 2.0))
    grad = np.zeros((2000, 4, 2))
    grad[:, 3, 0] = np.exp(-(dist / 0.01) ** 2) + 0.01 * rng.random(2000)
    bundle = {"node_pos": pos, "primitives_grad": grad}
    arrays.update(shock_node_pos=pos, shock_grad_p=grad[:, 3, :])
    out["helpers"]["shock"] = {"upper": ns["_measure_shock_angle"](bundle, None, 1.5, 2.0, 1.0, 0.0875, 0.0, "upper"),
                               "lower": ns["_measure_shock_angle"](bundle, None, 1.5, 2.0, 1.0, 0.0875, 0.0, "lower")}
    rows = [{"h": h, "e": 0.3 * h ** 1.7 * (1 + 0.05 * rng.standard_normal())} for h in (0.2, 0.1, 0.05, 0.025, 0.0125)]
    p_ord, r2, npts = ns["fit_order"](rows, "e")
    out["helpers"]["fit"] = {"rows": rows, "p": p_ord, "r2": r2, "n": npts}
    vals = {h: 0.05 + 0.3 * h ** 1.8 + 0.01 * h ** 3 for h in ns["H_GCI"]}
    out["helpers"]["gci"] = {"values": {str(h): v for h, v in vals.items()}, "chain": ns["H_GCI"],
                             "triplets": ns["richardson_gci"](vals)}
    s_ref = np.linspace(0, 2, 50)
    ref_p = {"s": s_ref, "mach": 1.5 + 0.3 * np.sin(3 * s_ref)}
    cur_p = {"s": np.linspace(0.05, 1.9, 37), "mach": 1.5 + 0.31 * np.sin(3 * np.linspace(0.05, 1.9, 37))}
    arrays.update(perr_ref_s=ref_p["s"], perr_ref_mach=ref_p["mach"], perr_cur_s=cur_p["s"],
                  perr_cur_mach=cur_p["mach"])
    out["helpers"]["profile_error"] = ns["_relative_profile_error"](ref_p, cur_p)
    np.savez_compressed(HERE / "reference_theory_inputs.npz", **arrays)
    for mach, aoa in ((1.5, 0.0), (2.0, 0.0), (2.0, 3.0), (2.5, 5.0), (3.0, -2.0), (1.05, 0.0)):
        panels = ns["diamond_panels"](mach, aoa, 5.0)
        out["panels"].append({"mach": mach, "aoa": aoa, "attached": bool(ns["all_attached"](panels)),
                    "panels": {k: {"M": p.M, "p_ratio": p.p_ratio_freestream, "Cp": p.Cp, "beta_deg": p.beta_deg,
                                   "attached": p.attached, "regime": p.regime} for k, p in panels.items()}})
    return out


def _summaries(utils_py: Path) -> list:
    """Run the reference's two summary functions, compiled from their source
    text, on a few argument sets; the file export goes to a scratch folder
    beside this script that is removed afterwards."""
    import ast
    import shutil
    tree = ast.parse(utils_py.read_text())
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef)
            and n.name in ("build_run_summary", "export_run_summary")]
    ns = {"np": np, "json": json, "Path": Path}
    exec(compile(ast.Module(body=keep, type_ignores=[]), str(utils_py), "exec"), ns)
    mesh = type("M", (), {"metadata": {"h": 0.025}, "tris": np.zeros((1234, 3), np.int32)})()
    cfg = dict(case="naca0012", Mach=0.8, aoa=-2.5, time_scheme="SRK2", flux="HLLC", reconstruction="MUSCL",
               mesh_path="m.npy", stationarity_threshold=1e-5, stationarity_check_every=25)
    calls = [dict(cd=0.0123, cl=-0.2, delta_s=1.5e-3, wall_time_s=2.25),
             dict(cd=0.0123, cl=-0.2, delta_s=1.5e-3, wall_time_s=2.25, stationarity_rel=3e-6, converged=True,
                  stopping_step=4200, compile_time_s=0.0, solve_time_s=2.25, stationarity_patience=3,
                  engineering_converged=False, engineering_stopping_step=5000, engineering_target_cd=0.0125,
                  engineering_target_cl=-0.21)]
    out = []
    scratch = HERE / "_summary_scratch"
    for kw in calls:
        summ = ns["build_run_summary"](cfg, mesh, **kw)
        ns["export_run_summary"]({"res": scratch}, summ, "AOA-2.50_M0.80_HLLC_MUSCL_SRK2_t1.00", verbose=False)
        f = scratch / "summary_AOA-2.50_M0.80_HLLC_MUSCL_SRK2_t1.00.json"
        out.append({"kwargs": kw, "summary": summ, "file": f.name, "text": f.read_text()})
    shutil.rmtree(scratch)
    return out


def mesh_digest(mesh) -> str:
    """sha256 of the mesh arrays the solver reads (the fixture's mesh identity)."""
    import hashlib
    h = hashlib.sha256()
    for a in (mesh.points, mesh.tris, mesh.neighbors, mesh.faces, mesh.face_markers, mesh.face_connectivity):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def hr_fixture(ref_root: str) -> Path:
    """The reference's own solver source on the HR diamond (h = 0.025, made by the package's mesher: 19,384 cells), M 2.0,
    alpha 0, CFL 0.6: 20 SRK2 steps in float32 and float64 with their dt,
    into ``reference_solver_hr.npz`` with the mesh's digest."""
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(HERE))
    sys.dont_write_bytecode = True
    import reference_solver_run as RS
    from eulersr_b200.meshing.generate import cached_mesh
    sys.path.insert(0, str(Path(ref_root) / "euler"))
    import config as ref_config
    mesh = cached_mesh("diamond", 0.025)
    out = {"mesh_sha256": np.asarray(mesh_digest(mesh)), "n_cells": np.asarray(mesh.n_cells)}
    for dname, dtp in (("f32", np.float32), ("f64", np.float64)):
        W, dt_ = RS.run(ref_root, mesh, 2.0, 0.0, 20, dtp, ref_config._AOA_CASES_LC)
        out[f"{dname}_W20"] = W
        out[f"{dname}_dt"] = np.asarray(dt_, dtype=dtp)
    path = HERE / "reference_solver_hr.npz"
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if len(args) != 1:
        sys.exit("usage: python tests/golden/make_reference_fixtures.py <path of the EulerSR checkout> [--hr-only]")
    if "--hr-only" not in sys.argv:
        print(main(args[0]))
    print(hr_fixture(args[0]))
