"""Mesh-convergence campaign on the diamond from solver bundles, as
EulerSR's ``euler/postproc/mesh_convergence_diamond.py`` runs it.

For a few representative (Mach, AoA) points it reads the latest bundle of
each mesh level (``<raw-dir>/h<h>/AOA<aoa>/AOA<aoa>_M<mach>_*_t<t>.npz``, the
layout ``eulersr_b200.grid`` and ``eulersr_b200.main`` write), recomputes CD
and CL from the conserved field, measures the wall-Mach profile's relative
error against the finest level, and computes the observed order and the
fine-grid GCI (Roache, safety factor 1.25) on the sliding triplets of the
dyadic chain (``mesh_convergence_diamond.py:141-161``). Writes
``raw_values.csv`` and ``gci_summary.csv`` with the reference's columns; the
reference's per-point figures are not drawn (plotting is not part of this
package).

    python -m eulersr_b200.mesh_convergence --raw-dir data/raw/diamond \\
        --mesh-dir data/meshes --out-dir data/validation/mesh_convergence_diamond
"""
from __future__ import annotations

import argparse
import math
import re
from pathlib import Path

import numpy as np

from .mesh import Mesh
from .postproc import force_coefficients, wall_profile

GAMMA = 1.4
# mesh_convergence_diamond.py:47-48: the full chain and its ratio-2 sub-chain
H_ALL = [0.4, 0.3, 0.2, 0.15, 0.1, 0.05, 0.025, 0.0175, 0.0125]
H_GCI = [0.4, 0.2, 0.1, 0.05, 0.025, 0.0125]
# mesh_convergence_diamond.py:51-59: (label, Mach, AoA)
TEST_POINTS = [
    ("P1_transsonique", 0.90, 0.0),
    ("P2_supersonique_marginal", 1.05, 0.0),
    ("P3_supersonique_propre", 1.50, 0.0),
    ("P4_supersonique_fort", 2.50, 0.0),
    ("P5_incidence", 2.00, 3.0),
    ("P6_mach2_symetrique", 2.00, 0.0),
    ("P7_incidence_forte", 2.50, 5.0),
]
_NAME = re.compile(r"AOA([+-]?[0-9.]+)_M([0-9.]+)_.*_t([0-9.]+)\.npz$")


def format_h(h: float) -> str:
    return f"h{h:.4f}".rstrip("0").rstrip(".")


def find_bundle(raw_dir, h: float, mach: float, aoa: float):
    """The bundle of (h, Mach, AoA) with the latest time stamp, or None."""
    d = Path(raw_dir) / format_h(h) / f"AOA{aoa:.2f}"
    if not d.exists():
        return None
    best, best_t = None, -1.0
    for f in d.glob(f"AOA{aoa:.2f}_M{mach:.2f}_*.npz"):
        m = _NAME.search(f.name)
        if m and float(m.group(3)) > best_t:
            best, best_t = f, float(m.group(3))
    return best


def load_level_mesh(mesh_dir, case: str, h: float) -> Mesh:
    """``<case>_h<h>.npz`` (this package's mesher) or the reference's ``.npy``."""
    for suffix in (".npz", ".npy"):
        p = Path(mesh_dir) / f"{case}_h{h}{suffix}"
        if p.exists():
            return Mesh.load(p)
    raise FileNotFoundError(f"no mesh {case}_h{h}.npz/.npy in {mesh_dir}")


def relative_profile_error(ref, cur, n_samples=400):
    """||Mach_cur - Mach_ref|| / ||Mach_ref|| on a common arc-length grid
    (mesh_convergence_diamond.py:106-119)."""
    if ref is None or cur is None or ref["s"].size < 2 or cur["s"].size < 2:
        return None
    lo, hi = max(ref["s"].min(), cur["s"].min()), min(ref["s"].max(), cur["s"].max())
    if hi <= lo:
        return None
    grid = np.linspace(lo, hi, n_samples)
    r = np.interp(grid, ref["s"], ref["mach"])
    c = np.interp(grid, cur["s"], cur["mach"])
    den = np.linalg.norm(r)
    return None if den <= 1e-16 else float(np.linalg.norm(c - r) / den)


def richardson_gci(values_by_h, chain=H_GCI, safety=1.25):
    """Observed order p = ln((f1-f2)/(f2-f3))/ln r and the fine-grid GCI
    safety |(f3-f2)/f3| / (r^p - 1) in percent on every sliding triplet
    (coarse, mid, fine) of ``chain`` (constant ratio r); a triplet whose
    differences vanish or change sign gets None."""
    r = chain[0] / chain[1]
    out = []
    for i in range(len(chain) - 2):
        h1, h2, h3 = chain[i], chain[i + 1], chain[i + 2]
        f1, f2, f3 = values_by_h.get(h1), values_by_h.get(h2), values_by_h.get(h3)
        if f1 is None or f2 is None or f3 is None:
            continue
        num, den = f1 - f2, f2 - f3
        if abs(den) < 1e-14 or num / den <= 0:
            out.append(dict(h_coarse=h1, h_mid=h2, h_fine=h3, p_obs=None, extrap=None, gci_fine_pct=None))
            continue
        p = math.log(num / den) / math.log(r)
        extrap = f3 + (f3 - f2) / (r ** p - 1.0)
        eps = abs((f3 - f2) / f3) if f3 != 0 else float("nan")
        out.append(dict(h_coarse=h1, h_mid=h2, h_fine=h3, p_obs=p, extrap=extrap,
                        gci_fine_pct=safety * eps / (r ** p - 1.0) * 100.0))
    return out


def run_point(raw_dir, mesh_dir, case, mach, aoa, h_all=H_ALL):
    """One row per mesh level that has a bundle: cells, CD, CL and the wall
    profile error against the finest level of ``h_all``."""
    meshes = {}

    def mesh(h):
        if h not in meshes:
            meshes[h] = load_level_mesh(mesh_dir, case, h)
        return meshes[h]

    ref = None
    fb = find_bundle(raw_dir, min(h_all), mach, aoa)
    if fb is not None:
        with np.load(fb) as d:
            ref = wall_profile(mesh(min(h_all)), d["conservatives"], GAMMA)
    rows = []
    for h in h_all:
        b = find_bundle(raw_dir, h, mach, aoa)
        if b is None:
            continue
        with np.load(b) as d:
            W = np.asarray(d["conservatives"], np.float64)
        m = mesh(h)
        cd, cl = force_coefficients(m, W, mach, GAMMA)
        prof = wall_profile(m, W, GAMMA)
        rows.append(dict(h=h, mach=mach, aoa=aoa, n_cells=m.n_cells, cd=cd, cl=cl, wall_profile=prof,
                         wall_profile_rel_err=relative_profile_error(ref, prof) if ref is not None else None))
    return rows


def campaign(raw_dir, mesh_dir, out_dir, case="diamond", points=TEST_POINTS, h_all=H_ALL, h_gci=H_GCI):
    """Every test point: the raw rows and the GCI triplets of CD and CL,
    written as raw_values.csv and gci_summary.csv in ``out_dir``."""
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    raw = ["label,mach,aoa,h,n_cells,cd,cl,wall_profile_rel_err"]
    summary = ["label,mach,aoa,h_coarse,h_mid,h_fine,quantity,p_obs,extrap,gci_fine_pct"]
    fmt = lambda v, f: "" if v is None else format(v, f)   # noqa: E731
    for label, mach, aoa in points:
        rows = run_point(raw_dir, mesh_dir, case, mach, aoa, h_all)
        for r in rows:
            raw.append(f"{label},{mach},{aoa},{r['h']},{r['n_cells']},{r['cd']:.6f},{r['cl']:.6f},"
                       f"{fmt(r['wall_profile_rel_err'], '.6e')}")
        by_h = {r["h"]: r for r in rows}
        for q in ("cd", "cl"):
            vals = {h: by_h[h][q] for h in h_gci if h in by_h}
            if len(vals) < 3:
                continue
            for t in richardson_gci(vals, h_gci):
                summary.append(f"{label},{mach},{aoa},{t['h_coarse']},{t['h_mid']},{t['h_fine']},{q},"
                               f"{fmt(t['p_obs'], '.6f')},{fmt(t['extrap'], '.6f')},{fmt(t['gci_fine_pct'], '.6f')}")
    (out_dir / "raw_values.csv").write_text("\n".join(raw) + "\n")
    (out_dir / "gci_summary.csv").write_text("\n".join(summary) + "\n")
    return out_dir / "raw_values.csv", out_dir / "gci_summary.csv"


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--case", default="diamond")
    ap.add_argument("--raw-dir", default=None)
    ap.add_argument("--mesh-dir", default=str(Path("data") / "meshes"))
    ap.add_argument("--out-dir", default=None)
    a = ap.parse_args(argv)
    raw_dir = a.raw_dir or str(Path("data") / "raw" / a.case)
    out_dir = a.out_dir or str(Path("data") / "validation" / f"mesh_convergence_{a.case}")
    for p in campaign(raw_dir, a.mesh_dir, out_dir, case=a.case):
        print(f"CSV -> {p}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
