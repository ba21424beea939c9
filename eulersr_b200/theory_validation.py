"""Shock-expansion validation campaigns on the diamond from solver bundles, as
EulerSR's ``euler/postproc/theory_validation_diamond.py`` runs them.

Each flat face of the diamond is a shock or an isentropic expansion in
cascade from upstream (front faces turn the flow by eps -/+ alpha, the
mid-chord shoulders expand it by 2 eps). Two campaigns, ``--campaign``:

* ``theory``: on the finest mesh, the solution's CD and CL against the
  theory's (the theoretical face pressures placed on the same wall cells and
  integrated with the same force routine), and per face the plateau Cp and
  Mach of the wall profile and the leading-edge shock angle measured in the
  field, against theory (``theory_vs_fvm.csv``).
* ``wall``: over the whole mesh chain, the errors of CD, CL, plateau Cp, the
  full wall-Cp profile, plateau Mach, the Mach maximum near the body and the
  shock angle, and the order of each fitted by a log-log regression over
  h <= 0.1 (``wall_profile_errors.csv``, ``wall_profile_order_fit.csv``).

Points whose front shocks would detach are skipped, as the reference does.
Bundles are found as ``eulersr_b200.mesh_convergence`` finds them; figures are
not drawn (plotting is not part of this package).

    python -m eulersr_b200.theory_validation --campaign both --raw-dir data/raw/diamond \\
        --mesh-dir data/meshes --out-root data/validation
"""
from __future__ import annotations

import argparse
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .mesh_convergence import H_ALL, find_bundle, load_level_mesh
from .postproc import _primitives, expansion, force_coefficients, turn

GAMMA = 1.4
P_INF = 1.0
RHO_INF = 1.0
H_REF = 0.0125                        # finest level of the chain
# theory_validation_diamond.py:186-203: shock search window and body window
SHOCK_WINDOW_X = (-0.35, 0.45)        # chords, from the leading edge
SHOCK_WINDOW_Y_FACTOR = 3.0           # in units of the diamond's height
SHOCK_TOP_PCT = 97.0                  # |grad p| percentile taken as shock points
OBJECT_WINDOW_X_FACTOR = 0.6
OBJECT_WINDOW_Y_FACTOR = 4.0
VALIDATION_POINTS = [
    ("P2_supersonique_marginal", 1.05, 0.0),
    ("P3_supersonique_propre", 1.50, 0.0),
    ("P4_supersonique_fort", 2.50, 0.0),
    ("P5_incidence", 2.00, 3.0),
    ("P6_mach2_symetrique", 2.00, 0.0),
    ("P7_incidence_forte", 2.50, 5.0),
]
PANEL_NAMES = ("upper_front", "upper_rear", "lower_front", "lower_rear")


@dataclass
class Panel:
    name: str
    deflection_deg: float     # local turning, + = compression
    regime: str               # "shock" or "expansion"
    attached: bool
    M: float
    p_ratio_freestream: float
    Cp: float
    beta_deg: float | None    # shock angle to the panel's upstream flow


def diamond_panels(mach, alpha_deg, eps_deg, gamma=GAMMA) -> dict:
    """The four faces' states (theory_validation_diamond.py:129-170): front
    faces turned by eps - alpha (upper) and eps + alpha (lower), rear faces
    expanded by 2 eps from the front state; Cp on the freestream. A front
    shock beyond the maximum deflection is marked detached."""
    eps, a = math.radians(eps_deg), math.radians(alpha_deg)
    q = 0.5 * gamma * mach * mach

    def side(defl):
        try:
            M1, r1, beta = turn(mach, defl, gamma)
        except ValueError:             # detached shock
            return None
        M2, r2 = expansion(M1, 2.0 * eps, gamma)
        return (M1, r1, beta), (M2, r1 * r2)

    out = {}
    for name_f, name_r, defl in (("upper_front", "upper_rear", eps - a), ("lower_front", "lower_rear", eps + a)):
        s = side(defl)
        if s is None:
            nan = float("nan")
            out[name_f] = Panel(name_f, math.degrees(defl), "shock", False, nan, nan, nan, None)
            out[name_r] = Panel(name_r, -2 * eps_deg, "expansion", False, nan, nan, nan, None)
            continue
        (M1, r1, beta), (M2, r2) = s
        out[name_f] = Panel(name_f, math.degrees(defl), "shock" if defl > 0 else "expansion", True, M1, r1,
                            (r1 - 1.0) / q, None if beta is None else math.degrees(beta))
        out[name_r] = Panel(name_r, -2 * eps_deg, "expansion", True, M2, r2, (r2 - 1.0) / q, None)
    return out


def all_attached(panels) -> bool:
    return all(p.attached for p in panels.values())


def panel_of(x, y, cx, cy) -> str:
    """Face of the diamond a wall point belongs to (theory_validation_diamond.py:237-244)."""
    if x < cx:
        return "upper_front" if y >= cy else "lower_front"
    return "upper_rear" if y >= cy else "lower_rear"


def _first_owner(mesh):
    """Flat (cell * 3 + slot) index of the first cell listing each face."""
    fc = mesh.face_connectivity.reshape(-1)
    first = np.full(mesh.n_faces, -1, np.int64)
    order = np.argsort(fc, kind="stable")
    fcs = fc[order]
    starts = np.r_[0, np.nonzero(np.diff(fcs))[0] + 1]
    first[fcs[starts]] = order[starts]
    return first


def side_wall_profile(mesh, W, side: str):
    """Pressure and Mach along the upper or lower wall (theory_validation_diamond.py:247-280):
    force-marker faces on that side of the domain's mid-height, sorted by
    midpoint x then y, valued at their first listing cell."""
    mid = mesh.face_midpoints()
    y_mid = 0.5 * (mesh.points[:, 1].min() + mesh.points[:, 1].max())
    on_side = mid[:, 1] <= y_mid if side == "lower" else mid[:, 1] >= y_mid
    ids = np.nonzero((mesh.face_markers == mesh.force_marker()) & on_side)[0]
    if ids.size == 0:
        return None
    ids = ids[np.lexsort((mid[ids, 1], mid[ids, 0]))]
    first = _first_owner(mesh)[ids]
    ids, cells = ids[first >= 0], first[first >= 0] // 3
    rho, u, v, p = _primitives(W, GAMMA)
    mach = np.hypot(u, v) / np.sqrt(np.abs(GAMMA * p / rho))
    return dict(x=mid[ids, 0], y=mid[ids, 1], p=p[cells], mach=mach[cells])


def panel_masks(profile, cx, cy):
    x, y = profile["x"], profile["y"]
    return {"upper_front": (x < cx) & (y >= cy), "upper_rear": (x >= cx) & (y >= cy),
            "lower_front": (x < cx) & (y < cy), "lower_rear": (x >= cx) & (y < cy)}


def plateau_value(profile, masks, key, transform, margin_frac=0.15):
    """Per face, the mean of transform(profile[key]) without the points within
    ``margin_frac`` of either end (theory_validation_diamond.py:283-299)."""
    out = {}
    for name, m in masks.items():
        xs, vals = profile["x"][m], profile[key][m]
        if xs.size < 3:
            out[name] = None
            continue
        vals = vals[np.argsort(xs, kind="stable")]
        n = xs.size
        lo, hi = int(n * margin_frac), int(n * (1 - margin_frac))
        if hi - lo < 1:
            lo, hi = 0, n
        out[name] = float(np.mean(transform(vals[lo:hi])))
    return out


def measure_shock_angle(node_pos, grad_p, cx, cy, chord, height, alpha_deg, side):
    """Leading-edge shock angle from the field (theory_validation_diamond.py:311-342):
    in a window from upstream of the leading edge to before mid-chord and up to
    3 heights off the axis, the cells in the top 3 % of |grad p| are taken as
    the shock; their principal direction (SVD) against the freestream
    direction gives the angle in degrees, or None with too few points."""
    pos = np.asarray(node_pos, np.float64)
    g = np.linalg.norm(np.asarray(grad_p, np.float64), axis=1)
    x_le = cx - chord / 2.0
    x_lo, x_hi = x_le + SHOCK_WINDOW_X[0] * chord, x_le + SHOCK_WINDOW_X[1] * chord
    if side == "upper":
        ym = (pos[:, 1] > cy + 0.005) & (pos[:, 1] < cy + SHOCK_WINDOW_Y_FACTOR * height)
    else:
        ym = (pos[:, 1] < cy - 0.005) & (pos[:, 1] > cy - SHOCK_WINDOW_Y_FACTOR * height)
    win = (pos[:, 0] > x_lo) & (pos[:, 0] < x_hi) & ym
    if win.sum() < 10:
        return None
    pts, gs = pos[win], g[win]
    sel = gs >= np.percentile(gs, SHOCK_TOP_PCT)
    if sel.sum() < 5:
        return None
    P = pts[sel] - pts[sel].mean(axis=0)
    direction = np.linalg.svd(P)[2][0]
    a = math.radians(alpha_deg)
    c = abs(float(direction @ np.array([math.cos(a), math.sin(a)])))
    return math.degrees(math.acos(min(1.0, max(-1.0, c))))


def theory_forces(mesh, panels, mach, cx, cy):
    """CD, CL of the theory on this mesh (theory_validation_diamond.py:345-372):
    the freestream pressure everywhere except the wall cells, which get their
    face's theoretical pressure (faces in index order, a later face of the
    same cell wins), integrated by the same routine as the solution."""
    p = np.full(mesh.n_cells, P_INF)
    mid = mesh.face_midpoints()
    first = _first_owner(mesh)
    for f in np.nonzero(mesh.face_markers == mesh.force_marker())[0]:
        if first[f] < 0:
            continue
        p[first[f] // 3] = P_INF * panels[panel_of(mid[f, 0], mid[f, 1], cx, cy)].p_ratio_freestream
    W = np.zeros((mesh.n_cells, 4))
    W[:, 0] = RHO_INF
    W[:, 3] = p / (GAMMA - 1.0)
    return force_coefficients(mesh, W, mach, GAMMA, RHO_INF, P_INF)


def _geometry(mesh):
    md = mesh.metadata
    return (float(md["center"]["cx"]), float(md["center"]["cy"]), float(md["chord"]), float(md["height"]))


def _eps_deg(mesh):
    _, _, chord, height = _geometry(mesh)
    return math.degrees(math.atan(height / chord))


def run_point(raw_dir, mesh_dir, case, label, mach, aoa, h=H_REF, eps_deg=None):
    """Campaign "theory" for one point on mesh level h; None when a front
    shock detaches or the bundle is missing."""
    bundle = find_bundle(raw_dir, h, mach, aoa)
    if bundle is None:
        return None
    mesh = load_level_mesh(mesh_dir, case, h)
    panels = diamond_panels(mach, aoa, _eps_deg(mesh) if eps_deg is None else eps_deg)
    if not all_attached(panels):
        return None
    cx, cy, chord, height = _geometry(mesh)
    with np.load(bundle) as d:
        W = np.asarray(d["conservatives"], np.float64)
        pos, gp = np.asarray(d["node_pos"]), np.asarray(d["primitives_grad"])[:, 3, :]
    cd, cl = force_coefficients(mesh, W, mach, GAMMA, RHO_INF, P_INF)
    cd_t, cl_t = theory_forces(mesh, panels, mach, cx, cy)
    q = 0.5 * RHO_INF * (mach * math.sqrt(GAMMA * P_INF / RHO_INF)) ** 2
    cp, mp = {}, {}
    for side in ("lower", "upper"):
        prof = side_wall_profile(mesh, W, side)
        if prof is None:
            continue
        masks = panel_masks(prof, cx, cy)
        cp.update({k: v for k, v in plateau_value(prof, masks, "p", lambda p: (p - P_INF) / q).items() if v is not None})
        mp.update({k: v for k, v in plateau_value(prof, masks, "mach", lambda m: m).items() if v is not None})
    beta = {"upper_front": measure_shock_angle(pos, gp, cx, cy, chord, height, aoa, "upper"),
            "lower_front": measure_shock_angle(pos, gp, cx, cy, chord, height, aoa, "lower")}
    rows = [(n, cp.get(n), panels[n].Cp, mp.get(n), panels[n].M, beta.get(n), panels[n].beta_deg, panels[n].regime)
            for n in PANEL_NAMES]
    return dict(label=label, mach=mach, aoa=aoa, cd_fvm=cd, cd_theory=cd_t, cl_fvm=cl, cl_theory=cl_t, panels=rows)


def compute_errors(raw_dir, mesh_dir, case, mach, aoa, h_all=H_ALL, eps_deg=None):
    """Campaign "wall" for one point: the error measures per mesh level
    (theory_validation_diamond.py:509-606); None when a front shock detaches."""
    rows = []
    for h in h_all:
        bundle = find_bundle(raw_dir, h, mach, aoa)
        if bundle is None:
            continue
        mesh = load_level_mesh(mesh_dir, case, h)
        panels = diamond_panels(mach, aoa, _eps_deg(mesh) if eps_deg is None else eps_deg)
        if not all_attached(panels):
            return None
        cx, cy, chord, height = _geometry(mesh)
        with np.load(bundle) as d:
            W = np.asarray(d["conservatives"], np.float64)
            pos, gp = np.asarray(d["node_pos"]), np.asarray(d["primitives_grad"])[:, 3, :]
        cd, cl = force_coefficients(mesh, W, mach, GAMMA, RHO_INF, P_INF)
        cd_t, cl_t = theory_forces(mesh, panels, mach, cx, cy)
        q = 0.5 * RHO_INF * (mach * math.sqrt(GAMMA * P_INF / RHO_INF)) ** 2
        cp_err, m_err, full = [], [], []
        for side in ("lower", "upper"):
            prof = side_wall_profile(mesh, W, side)
            if prof is None:
                continue
            masks = panel_masks(prof, cx, cy)
            for n, v in plateau_value(prof, masks, "p", lambda p: (p - P_INF) / q).items():
                if v is not None:
                    cp_err.append(v - panels[n].Cp)
            for n, v in plateau_value(prof, masks, "mach", lambda m: m).items():
                if v is not None:
                    m_err.append(v - panels[n].M)
            cp_t = np.array([panels[panel_of(x, y, cx, cy)].Cp for x, y in zip(prof["x"], prof["y"])])
            full.append((prof["p"] - P_INF) / q - cp_t)
        if not cp_err or not full:
            continue
        rho, u, v, p = _primitives(W, GAMMA)
        mach_f = np.hypot(u, v) / np.sqrt(np.abs(GAMMA * p / rho))
        win = (np.abs(pos[:, 0] - cx) < OBJECT_WINDOW_X_FACTOR * chord) & \
              (np.abs(pos[:, 1] - cy) < OBJECT_WINDOW_Y_FACTOR * height)
        mach_max = float(mach_f[win].max()) if win.any() else float(mach_f.max())
        mach_max_t = max(pp.M for pp in panels.values())
        berr = []
        for side, n in (("upper", "upper_front"), ("lower", "lower_front")):
            b = measure_shock_angle(pos, gp, cx, cy, chord, height, aoa, side)
            if b is not None and panels[n].beta_deg is not None:
                berr.append(b - panels[n].beta_deg)
        rms = lambda e: float(np.sqrt(np.mean(np.square(e))))   # noqa: E731
        rows.append(dict(h=h, n_cells=mesh.n_cells, cd_fvm=cd, cd_theory=cd_t, err_cd=abs(cd - cd_t),
                         cl_fvm=cl, cl_theory=cl_t, err_cl=abs(cl - cl_t), rms_plateau=rms(cp_err),
                         rms_full=rms(np.concatenate(full)), rms_mach_plateau=rms(m_err) if m_err else None,
                         mach_max_fvm=mach_max, mach_max_theory=mach_max_t, err_mach_max=abs(mach_max_t - mach_max),
                         err_beta=rms(berr) if berr else None))
    return rows


def fit_order(rows, key, h_max=0.1):
    """Slope and R^2 of the least-squares line through log(error) against
    log(h) over the levels h <= h_max with a positive error (at least 3)."""
    pts = [(r["h"], r[key]) for r in rows if r["h"] <= h_max and r[key] is not None and r[key] > 0]
    if len(pts) < 3:
        return None, None, len(pts)
    lh = np.log([p[0] for p in pts])
    le = np.log([p[1] for p in pts])
    slope, icpt = np.polyfit(lh, le, 1)
    ss_res = float(np.sum((le - (slope * lh + icpt)) ** 2))
    ss_tot = float(np.sum((le - le.mean()) ** 2))
    return float(slope), (1.0 - ss_res / ss_tot if ss_tot > 0 else float("nan")), len(pts)


def _f(v, spec):
    return "" if v is None else format(v, spec)


def run_theory_validation(raw_dir, mesh_dir, out_dir, case="diamond", points=VALIDATION_POINTS, h=H_REF):
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    lines = ["label,mach,aoa,Cd_fvm,Cd_theory,Cl_fvm,Cl_theory,panel,"
             "Cp_fvm,Cp_theory,M_fvm,M_theory,beta_fvm_deg,beta_theory_deg,regime"]
    for label, mach, aoa in points:
        r = run_point(raw_dir, mesh_dir, case, label, mach, aoa, h)
        if r is None:
            continue
        for n, cpf, cpt, mf, mt, bf, bt, reg in r["panels"]:
            lines.append(f"{label},{mach},{aoa},{r['cd_fvm']:.6f},{r['cd_theory']:.6f},{r['cl_fvm']:.6f},"
                         f"{r['cl_theory']:.6f},{n},{_f(cpf, '.6f')},{cpt:.6f},{_f(mf, '.6f')},{mt:.6f},"
                         f"{_f(bf, '.4f')},{_f(bt, '.4f')},{reg}")
    path = out_dir / "theory_vs_fvm.csv"
    path.write_text("\n".join(lines) + "\n")
    return path


def run_wall_convergence(raw_dir, mesh_dir, out_dir, case="diamond", points=VALIDATION_POINTS, h_all=H_ALL,
                         h_max=0.1):
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    csv = ["label,mach,aoa,h,n_cells,cd_fvm,cd_theory,err_cd,cl_fvm,cl_theory,err_cl,"
           "rms_cp_plateau,rms_cp_profil_complet,"
           "rms_mach_plateau,mach_max_fvm,mach_max_theory,err_mach_max,rms_err_beta_deg"]
    summary = ["label,mach,aoa,quantity,p_order,r2,n_points"]
    for label, mach, aoa in points:
        rows = compute_errors(raw_dir, mesh_dir, case, mach, aoa, h_all)
        if rows is None:
            continue
        for r in rows:
            csv.append(f"{label},{mach},{aoa},{r['h']},{r['n_cells']},{r['cd_fvm']:.6f},{r['cd_theory']:.6f},"
                       f"{r['err_cd']:.6e},{r['cl_fvm']:.6f},{r['cl_theory']:.6f},{r['err_cl']:.6e},"
                       f"{r['rms_plateau']:.6e},{r['rms_full']:.6e},{_f(r['rms_mach_plateau'], '.6e')},"
                       f"{r['mach_max_fvm']:.6f},{r['mach_max_theory']:.6f},{r['err_mach_max']:.6e},"
                       f"{_f(r['err_beta'], '.6e')}")
        for key, tag in (("err_cd", "cd"), ("err_cl", "cl"), ("rms_plateau", "cp_plateau"),
                         ("rms_full", "cp_profil_complet"), ("rms_mach_plateau", "mach_plateau"),
                         ("err_mach_max", "mach_max"), ("err_beta", "beta_choc")):
            p, r2, n = fit_order(rows, key, h_max)
            if p is not None:
                summary.append(f"{label},{mach},{aoa},{tag},{p:.6f},{r2:.6f},{n}")
    a, b = out_dir / "wall_profile_errors.csv", out_dir / "wall_profile_order_fit.csv"
    a.write_text("\n".join(csv) + "\n")
    b.write_text("\n".join(summary) + "\n")
    return a, b


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--case", default="diamond")
    ap.add_argument("--campaign", default="both", choices=["theory", "wall", "both"])
    ap.add_argument("--raw-dir", default=None)
    ap.add_argument("--mesh-dir", default=str(Path("data") / "meshes"))
    ap.add_argument("--out-root", default=str(Path("data") / "validation"))
    a = ap.parse_args(argv)
    raw = a.raw_dir or str(Path("data") / "raw" / a.case)
    if a.campaign in ("theory", "both"):
        print(f"CSV -> {run_theory_validation(raw, a.mesh_dir, Path(a.out_root) / f'theory_{a.case}', a.case)}")
    if a.campaign in ("wall", "both"):
        for p in run_wall_convergence(raw, a.mesh_dir, Path(a.out_root) / f"wall_profile_convergence_{a.case}",
                                      a.case):
            print(f"CSV -> {p}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
