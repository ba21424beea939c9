"""Validation of diamond-airfoil solutions against shock-expansion theory.

The reference validates its solver against the analytic supersonic flow over
a diamond (``euler/postproc/theory_validation_diamond.py``): oblique shocks
(or Prandtl-Meyer expansions) on the front faces, Prandtl-Meyer expansions
over the shoulders, the resulting face pressures, the pressure-force
coefficients in body axes, and the leading-edge shock angle measured from the
computed field. The relations below are the textbook ones (theta-beta-Mach,
normal-shock jumps, Prandtl-Meyer function), solved numerically.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _bisect(f, a, b, tol=1e-14, it=200):
    fa = f(a)
    for _ in range(it):
        m = 0.5 * (a + b)
        fm = f(m)
        if (fm > 0) == (fa > 0):
            a, fa = m, fm
        else:
            b = m
        if b - a < tol:
            break
    return 0.5 * (a + b)


def theta_from_beta(M, beta, g=1.4):
    """Flow deflection behind an oblique shock of angle beta."""
    num = 2.0 / math.tan(beta) * (M * M * math.sin(beta) ** 2 - 1.0)
    den = M * M * (g + math.cos(2.0 * beta)) + 2.0
    return math.atan(num / den)


def oblique_shock_beta(M, theta, g=1.4):
    """Weak-solution shock angle for deflection theta (radians)."""
    mu = math.asin(1.0 / M)
    # the deflection is maximal at beta_max; the weak branch lies in (mu, beta_max)
    bs = np.linspace(mu + 1e-9, math.pi / 2 - 1e-9, 4001)
    th = np.array([theta_from_beta(M, b, g) for b in bs])
    i = int(np.argmax(th))
    if theta > th[i]:
        raise ValueError(f"detached shock: deflection {math.degrees(theta):.2f} deg above max "
                         f"{math.degrees(th[i]):.2f} deg at M={M}")
    return _bisect(lambda b: theta_from_beta(M, b, g) - theta, mu + 1e-12, float(bs[i]))


def oblique_shock(M, theta, g=1.4):
    """(beta, M2, p2/p1) for deflection theta."""
    beta = oblique_shock_beta(M, theta, g)
    mn1 = M * math.sin(beta)
    pr = 1.0 + 2.0 * g / (g + 1.0) * (mn1 * mn1 - 1.0)
    mn2 = math.sqrt((1.0 + 0.5 * (g - 1.0) * mn1 * mn1) / (g * mn1 * mn1 - 0.5 * (g - 1.0)))
    return beta, mn2 / math.sin(beta - theta), pr


def prandtl_meyer(M, g=1.4):
    a = math.sqrt((g + 1.0) / (g - 1.0))
    return a * math.atan(math.sqrt((M * M - 1.0) / (a * a))) - math.atan(math.sqrt(M * M - 1.0))


def expansion(M, dtheta, g=1.4):
    """(M2, p2/p1) after turning the flow away by dtheta (radians) isentropically."""
    nu2 = prandtl_meyer(M, g) + dtheta
    M2 = _bisect(lambda m: prandtl_meyer(m, g) - nu2, 1.0 + 1e-12, 100.0)
    pr = ((1.0 + 0.5 * (g - 1.0) * M * M) / (1.0 + 0.5 * (g - 1.0) * M2 * M2)) ** (g / (g - 1.0))
    return M2, pr


def turn(M, delta, g=1.4):
    """Compression (shock) for delta > 0, expansion for delta < 0: (M2, p2/p1, beta or None)."""
    if delta > 0:
        beta, M2, pr = oblique_shock(M, delta, g)
        return M2, pr, beta
    if delta < 0:
        M2, pr = expansion(M, -delta, g)
        return M2, pr, None
    return M, 1.0, None


@dataclass
class DiamondTheory:
    cd: float
    cl: float
    p_faces: dict          # pressure on upper/lower front/rear faces (freestream p = p_inf)
    mach_faces: dict
    beta_upper_deg: float | None
    beta_lower_deg: float | None


def diamond_theory(M, alpha_deg=0.0, half_angle_deg=5.0, g=1.4, p_inf=1.0) -> DiamondTheory:
    """Shock-expansion solution of a symmetric diamond of half angle eps at
    incidence alpha; coefficients in body axes with the reference's
    convention (fluid-cell outward normals, q = 1/2 gamma p M^2, chord 1)."""
    eps = math.radians(half_angle_deg)
    a = math.radians(alpha_deg)
    Mu1, pu1, bu = turn(M, eps - a, g)
    Ml1, pl1, bl = turn(M, eps + a, g)
    Mu2, pu2 = expansion(Mu1, 2 * eps, g)
    Ml2, pl2 = expansion(Ml1, 2 * eps, g)
    p = {"upper_front": pu1 * p_inf, "upper_rear": pu1 * pu2 * p_inf,
         "lower_front": pl1 * p_inf, "lower_rear": pl1 * pl2 * p_inf}
    q = 0.5 * g * p_inf * M * M
    L = 0.5 / math.cos(eps)               # face length for chord 1
    s, c = math.sin(eps), math.cos(eps)
    cd = L / q * (s * p["upper_front"] - s * p["upper_rear"] + s * p["lower_front"] - s * p["lower_rear"])
    cl = L / q * (-c * p["upper_front"] - c * p["upper_rear"] + c * p["lower_front"] + c * p["lower_rear"])
    return DiamondTheory(cd=cd, cl=cl, p_faces=p,
                         mach_faces={"upper_front": Mu1, "upper_rear": Mu2, "lower_front": Ml1, "lower_rear": Ml2},
                         beta_upper_deg=math.degrees(bu) if bu is not None else None,
                         beta_lower_deg=math.degrees(bl) if bl is not None else None)


def shock_angle_deg(mesh, W, le=(1.0, 2.0), chord=1.0, gamma=1.4, p_inf=1.0, x_range=(0.15, 0.45), side=+1):
    """Leading-edge shock angle measured from a solution: in vertical bands
    x - x_le in ``x_range`` (fractions of the chord) above (side=+1) or below
    the body, the shock sits where the pressure first crosses the mid level
    between the freestream and the post-shock plateau; a least-squares line
    through those points gives the angle to the freestream direction."""
    W = np.asarray(W, np.float64)
    rho = W[:, 0]
    u, v = W[:, 1] / rho, W[:, 2] / rho
    p = (W[:, 3] - 0.5 * rho * (u * u + v * v)) * (gamma - 1.0)
    xc, yc = mesh.barycenter[:, 0] - le[0], (mesh.barycenter[:, 1] - le[1]) * side
    pts = []
    for x0 in np.linspace(x_range[0], x_range[1], 12) * chord:
        band = (np.abs(xc - x0) < 0.02 * chord) & (yc > 0) & (yc < 0.8 * chord)
        if band.sum() < 8:
            continue
        ys, ps = yc[band], p[band]
        o = np.argsort(ys)
        ys, ps = ys[o], ps[o]
        p_post = np.median(ps[: max(3, len(ps) // 10)])
        mid = 0.5 * (p_post + p_inf)
        far = np.nonzero(ps < mid)[0]
        if len(far) == 0 or p_post <= p_inf * 1.001:
            continue
        j = far[0]
        if j == 0:
            continue
        y_cross = ys[j - 1] + (mid - ps[j - 1]) * (ys[j] - ys[j - 1]) / (ps[j] - ps[j - 1])
        pts.append((x0, y_cross))
    if len(pts) < 3:
        return float("nan")
    X, Y = np.asarray(pts).T
    slope = np.polyfit(X, Y, 1)[0]
    return math.degrees(math.atan(slope))


def _primitives(W, gamma=1.4):
    """Density, velocity and pressure of conserved rows (helper.py:25-36, M = 1)."""
    W = np.asarray(W, np.float64)
    rho = W[:, 0]
    u, v = W[:, 1] / rho, W[:, 2] / rho
    p = (W[:, 3] - 0.5 * rho * (u * u + v * v)) * (gamma - 1.0)
    return rho, u, v, p


def force_coefficients(mesh, W, mach, gamma=1.4, rho_inf=1.0, p_inf=1.0):
    """(CD, CL) of a field on the host, as helper.py:366-415 computes them:
    the owner cell's pressure (no reconstruction) times the owner's outward
    normal and the face length, summed over the force-marker faces, over
    0.5 rho U^2 L_ref in body axes, U = M sqrt(gamma p / rho)."""
    _, _, _, p = _primitives(W, gamma)
    faces, cells, slots = mesh.wall_owner_data()
    n = mesh.normals[cells, slots]
    ds = mesh.surface[faces]
    u_inf = mach * math.sqrt(gamma * p_inf / rho_inf)
    q = 0.5 * rho_inf * u_inf ** 2 * float(mesh.metadata.get("obstacle_length", 1.0) or 1.0)
    return float(np.sum(p[cells] * n[:, 0] * ds) / q), float(np.sum(p[cells] * n[:, 1] * ds) / q)


def wall_profile(mesh, W, gamma=1.4):
    """Wall Mach and pressure along the lower body surface (helper.py:439-506):
    wall faces whose midpoint lies at or below the domain's mid-height (all
    wall faces when none does), sorted by midpoint x then y, each valued at its
    first listing cell; ``s`` is the arc length along the sorted midpoints."""
    mid = mesh.face_midpoints()
    wall = np.isin(mesh.face_markers, mesh.wall_markers())
    empty = np.empty(0)
    if not wall.any():
        return {"s": empty, "x": empty, "y": empty, "mach": empty, "pressure": empty,
                "face_ids": np.empty(0, np.int32)}
    y_mid = 0.5 * float(mesh.points[:, 1].min() + mesh.points[:, 1].max())
    ids = np.nonzero(wall & (mid[:, 1] <= y_mid))[0]
    if ids.size == 0:
        ids = np.nonzero(wall)[0]
    ids = ids[np.lexsort((mid[ids, 1], mid[ids, 0]))]
    # first (cell, slot) listing each face, row-major, as the owner lookup does
    fc = mesh.face_connectivity.reshape(-1)
    first = np.full(mesh.n_faces, -1, np.int64)
    order = np.argsort(fc, kind="stable")
    fcs = fc[order]
    starts = np.r_[0, np.nonzero(np.diff(fcs))[0] + 1]
    first[fcs[starts]] = order[starts]
    keep = first[ids] >= 0
    ids = ids[keep]
    cells = first[ids] // 3
    rho, u, v, p = _primitives(W, gamma)
    a = np.sqrt(np.maximum(gamma * p[cells] / rho[cells], 1e-14))
    m = mid[ids]
    seg = np.linalg.norm(np.diff(m, axis=0), axis=1) if len(ids) > 1 else empty
    return {"s": np.concatenate(([0.0], np.cumsum(seg))) if len(ids) else empty, "x": m[:, 0], "y": m[:, 1],
            "mach": np.hypot(u[cells], v[cells]) / a, "pressure": p[cells], "face_ids": ids.astype(np.int32)}


def validate_diamond(h=0.025, machs=(1.5, 2.0), precision="f64"):
    """Converged diamond solves (alpha 0) against shock-expansion theory, as
    euler/postproc/theory_validation_diamond.py does: CD error and the
    leading-edge shock-angle error per Mach. Needs the GPU library."""
    import numpy as np
    from .meshing import build_mesh
    from .solver import FlowCase, Solver
    mesh = build_mesh("diamond", h)
    rows = []
    for M in machs:
        th = diamond_theory(M, 0.0, half_angle_deg=5.0)
        s = Solver(mesh, 1, precision=precision, threshold=1e-5, check_every=25)
        s.set_case(0, FlowCase(mach=M, aoa_deg=0.0, cfl=0.6, tf=30.0,
                               dtype=np.float64 if precision == "f64" else np.float32))
        r = s.run()[0]
        beta = shock_angle_deg(mesh, s.get_state(0), le=(1.0, 2.0))
        rows.append({"mach": M, "cells": mesh.n_cells, "converged": bool(r["converged"]), "steps": int(r["steps"]),
                     "cd": float(r["cd"]), "cd_theory": th.cd, "cd_err": abs(r["cd"] - th.cd) / th.cd,
                     "beta_deg": float(beta), "beta_theory_deg": th.beta_upper_deg,
                     "beta_err_deg": abs(beta - th.beta_upper_deg)})
        s.close()
    return rows


if __name__ == "__main__":
    import json
    import sys
    prec = sys.argv[1] if len(sys.argv) > 1 else "f64"
    for row in validate_diamond(precision=prec):
        print(json.dumps(row))
