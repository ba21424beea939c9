"""Run configuration: TOML defaults, CLI overrides, mesh loading, output dirs.

Same keys, flags and naming as the reference's ``euler/config.py:24-174`` so
that configurations and scripts carry over unchanged.
"""
from __future__ import annotations

import tomllib
from argparse import ArgumentParser
from copy import deepcopy
from pathlib import Path

DEFAULT_CONFIG_PATH = Path(__file__).with_name("config.toml")

# euler/config.py:15-21
AOA_CASES = ("diamond", "naca0012", "naca2412", "rae2822", "oneraD", "oa209", "diamond_tx", "diamond_txy",
             "diamond_alpha10", "rae2822_txy", "diamond_sym", "naca23012", "diamond_big", "cylinder")
KNOWN_CASES = ("bump",) + AOA_CASES
AOA_CASES_LC = tuple(c.lower() for c in AOA_CASES)
KNOWN_CASES_LC = tuple(c.lower() for c in KNOWN_CASES)


def load_default_config(config_path: str | Path | None = None) -> dict:
    path = Path(config_path) if config_path is not None else DEFAULT_CONFIG_PATH
    with path.open("rb") as fh:
        cfg = tomllib.load(fh)
    cfg["export"] = deepcopy(cfg.get("export", {}))
    return cfg


def build_config_from_cli(default_cfg: dict, argv=None) -> dict:
    """The CLI of euler/config.py:32-60 (plus --precision)."""
    p = ArgumentParser(description="Explicit 2-D Euler solve on B200")
    p.add_argument("--case", choices=KNOWN_CASES, default=default_cfg["case"])
    p.add_argument("--mach", type=float, default=default_cfg["Mach"])
    p.add_argument("--mesh-path", type=str, default=default_cfg["mesh_path"])
    p.add_argument("--time-scheme", choices=("EE", "RK2", "SRK2", "SSP_RK2"), default=default_cfg["time_scheme"])
    p.add_argument("--flux", choices=("Rusanov", "HLLC"), default=default_cfg["flux"])
    p.add_argument("--reconstruction", choices=("constant", "MUSCL", "muscl"), default=default_cfg["reconstruction"])
    p.add_argument("--aoa", type=float, default=default_cfg.get("aoa", 0.0))
    p.add_argument("--stationarity-threshold", type=float, default=default_cfg.get("stationarity_threshold", 1e-6))
    p.add_argument("--stationarity-check-every", type=int, default=default_cfg.get("stationarity_check_every", 25))
    p.add_argument("--stationarity-patience", type=int, default=default_cfg.get("stationarity_patience", 1))
    p.add_argument("--precision", choices=("f32", "f64"), default=default_cfg.get("precision"))
    p.add_argument("--verbose", dest="verbose", action="store_true", default=default_cfg.get("verbose", True))
    p.add_argument("--quiet", dest="verbose", action="store_false")
    a = p.parse_args(argv)
    cfg = deepcopy(default_cfg)
    cfg["case"] = a.case
    cfg["Mach"] = a.mach
    cfg["mesh_path"] = a.mesh_path
    cfg["time_scheme"] = "SRK2" if a.time_scheme == "SSP_RK2" else a.time_scheme
    cfg["flux"] = a.flux
    cfg["reconstruction"] = "MUSCL" if str(a.reconstruction).lower() == "muscl" else a.reconstruction
    cfg["aoa"] = float(a.aoa)
    cfg["stationarity_threshold"] = float(a.stationarity_threshold)
    cfg["stationarity_check_every"] = max(1, int(a.stationarity_check_every))
    cfg["stationarity_patience"] = max(1, int(a.stationarity_patience))
    if a.precision:
        cfg["precision"] = a.precision
    cfg["verbose"] = bool(a.verbose)
    return cfg


def load_mesh(cfg: dict):
    """euler/config.py:63-79: the reference's pickled .npy or an extended graph.npz."""
    from .mesh import Mesh
    if cfg.get("mesh_path") is None:
        raise ValueError("the mesh path must be given with --mesh-path or in the configuration")
    path = Path(cfg["mesh_path"])
    if not path.suffix:
        path = path.with_suffix(".npy")
    return Mesh.load(path)


def format_h(mesh) -> str:
    h = mesh.metadata.get("h", None)
    if h is None:
        return "h"
    return f"h{float(h):.4f}".rstrip("0").rstrip(".")


def format_condition_tag(cfg) -> str:
    mach = f"M{float(cfg.get('Mach')):.2f}"
    if str(cfg.get("case", "")).lower() in AOA_CASES_LC:
        return f"AOA{float(cfg.get('aoa', 0.0)):.2f}_{mach}"
    return mach


def format_snapshot_name(cfg, t) -> str:
    """euler/config.py:97-103."""
    return (f"{format_condition_tag(cfg)}_{str(cfg['flux']).upper()}_{str(cfg['reconstruction']).upper()}_"
            f"{str(cfg['time_scheme']).upper()}_t{t:.2f}")


def setup_dirs(cfg, mesh, root: str | Path = ".") -> dict:
    """euler/config.py:120-139 rooted at ``root``."""
    root = Path(root)
    h_dir = format_h(mesh)
    case = str(cfg.get("case", ""))
    if case.lower() in AOA_CASES_LC:
        tag = f"AOA{float(cfg.get('aoa', 0.0)):.2f}"
        dirs = {"fig": root / "euler" / "figures" / case / h_dir / tag, "res": root / "data" / "raw" / case / h_dir / tag}
    else:
        dirs = {"fig": root / "euler" / "figures" / case / h_dir, "res": root / "euler" / "results" / case / h_dir}
    for d in dirs.values():
        d.mkdir(parents=True, exist_ok=True)
    if cfg.get("verbose", True):
        print(f"Output : {dirs['res']}")
    return dirs
