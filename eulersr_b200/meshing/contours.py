"""Body contours and boundary sampling for the mesher.

The sampling rules and mesh-size functions follow the reference mesher so
that cell counts at a given ``h`` come out comparable:

* uniform sampling of each diamond side with ceil(len/h) points
  (``euler/meshing/diamond.py:20-29``);
* outer box sampled by stepping the local size function with a minimum step
  of h (``euler/meshing/mesh_utils.py:28-48,153-170``);
* airfoil surfaces sampled by Menger curvature, step clip(2 h_body / kappa,
  h/5, 2h/3) (``mesh_utils.py:59-111``);
* size functions growing with the distance to the body, faster upstream
  (``diamond.py:32-60``, ``mesh_utils.py:114-141``).

Airfoil shapes are the analytic NACA families: 4-digit thickness with the
closed-trailing-edge coefficient, 4-digit two-parabola camber, and the
5-digit (non-reflex) cubic camber line; the coefficients are the published
NACA report values.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.spatial import cKDTree


@dataclass(frozen=True)
class SizeParams:
    """Grading parameters (the reference's ``MeshSizeParams``,
    ``mesh_utils.py:19-25``)."""
    growth_rate: float = 0.09
    left_growth_rate: float = 0.23
    obstacle_factor: float = 0.0
    max_size_factor: float = 6.0
    left_margin_factor: float = 5.0


DIAMOND_SIZE = SizeParams(growth_rate=0.07, left_growth_rate=0.18)
AIRFOIL_SIZE = SizeParams()


def smoothstep(x):
    x = np.clip(x, 0.0, 1.0)
    return x * x * (3.0 - 2.0 * x)


def triangle_area_from_h(h):
    """Area of the equilateral triangle of side h."""
    return np.sqrt(3.0) * np.asarray(h) ** 2 / 4.0


def sample_segment(p0, p1, size_fn, min_step):
    """Points from p0 (included) towards p1 (excluded), each step the local size
    at the half-step point, never below ``min_step``; the last interval is
    merged when it would be shorter than half a minimum step."""
    p0 = np.asarray(p0, float)
    p1 = np.asarray(p1, float)
    d = p1 - p0
    L = float(np.linalg.norm(d))
    if L == 0.0:
        return np.empty((0, 2))
    u = d / L
    out = [p0]
    s = 0.0
    while s < L:
        mid = p0 + u * min(s + 0.5 * min_step, L)
        step = max(min_step, float(size_fn(mid)))
        nxt = min(L, s + step)
        if nxt >= L or (L - nxt) < 0.5 * min_step:
            break
        out.append(p0 + u * nxt)
        s = nxt
    return np.asarray(out)


def menger_curvature(pts):
    """Discrete curvature 2|cross|/(|ab||bc||ca|) at interior points, copied to
    the ends."""
    pts = np.asarray(pts, float)
    a, b, c = pts[:-2], pts[1:-1], pts[2:]
    cross = np.abs((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0]))
    den = np.linalg.norm(b - a, axis=1) * np.linalg.norm(c - b, axis=1) * np.linalg.norm(a - c, axis=1)
    k = np.zeros(len(pts))
    k[1:-1] = np.where(den > 1e-20, 2.0 * cross / np.where(den > 1e-20, den, 1.0), 0.0)
    k[0], k[-1] = k[1], k[-2]
    return k


def sample_half_contour(half, h_body, h_min):
    """Curvature-adaptive resampling of one airfoil surface."""
    arclen = np.r_[0.0, np.cumsum(np.linalg.norm(np.diff(half, axis=0), axis=1))]
    total = arclen[-1]
    n_uni = max(int(total / (0.5 * h_min)) + 1, 8)
    s_uni = np.linspace(0.0, total, n_uni)
    xy_uni = np.column_stack([np.interp(s_uni, arclen, half[:, 0]), np.interp(s_uni, arclen, half[:, 1])])
    kappa = menger_curvature(xy_uni)
    pts, s = [], 0.0
    while s < total:
        pts.append([np.interp(s, arclen, half[:, 0]), np.interp(s, arclen, half[:, 1])])
        k = max(float(np.interp(s, s_uni, kappa)), 1e-10)
        s += float(np.clip(h_body / k * 2, h_min, h_body))
    return np.asarray(pts)


# --------------------------------------------------------------------------
# NACA shapes
# --------------------------------------------------------------------------

def naca_thickness(xc, t):
    """4-digit half thickness, closed trailing edge (last coefficient -0.1036)."""
    xc = np.maximum(xc, 0.0)
    return 5 * t * (0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc ** 2 + 0.2843 * xc ** 3 - 0.1036 * xc ** 4)


def naca4_camber(xc, m, p):
    """Two-parabola 4-digit camber line and its slope."""
    if m == 0.0 or p == 0.0:
        return np.zeros_like(xc), np.zeros_like(xc)
    yc = np.where(xc < p, m / p ** 2 * (2 * p * xc - xc ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * xc - xc ** 2))
    dyc = np.where(xc < p, 2 * m / p ** 2 * (p - xc), 2 * m / (1 - p) ** 2 * (p - xc))
    return yc, dyc


# Non-reflex 5-digit camber constants (r, k1) by position of maximum camber,
# for a design lift coefficient of 0.3; scaled linearly for other CLi.
_NACA5_TABLE = {0.05: (0.0580, 361.400), 0.10: (0.1260, 51.640), 0.15: (0.2025, 15.957),
                0.20: (0.2900, 6.643), 0.25: (0.3910, 3.230)}


def naca5_camber(xc, cli, p):
    """5-digit cubic camber line: k1/6 (x^3 - 3 r x^2 + r^2 (3 - r) x) ahead of
    x=r and k1 r^3/6 (1 - x) behind it."""
    r, k1 = _NACA5_TABLE[round(p, 2)]
    k1 = k1 * cli / 0.3
    yc = np.where(xc < r, k1 / 6 * (xc ** 3 - 3 * r * xc ** 2 + r ** 2 * (3 - r) * xc), k1 * r ** 3 / 6 * (1 - xc))
    dyc = np.where(xc < r, k1 / 6 * (3 * xc ** 2 - 6 * r * xc + r ** 2 * (3 - r)), -k1 * r ** 3 / 6 * np.ones_like(xc))
    return yc, dyc


def naca_spec(name: str):
    """Parse 'naca0012', 'naca2412', 'naca23012' into a shape description."""
    digits = name.lower().replace('naca', '')
    if len(digits) == 4:
        return dict(kind='naca4', m=int(digits[0]) / 100.0, p=int(digits[1]) / 10.0, t=int(digits[2:]) / 100.0)
    if len(digits) == 5:
        if digits[2] != '0':
            raise ValueError("reflexed 5-digit sections are not supported")
        return dict(kind='naca5', cli=int(digits[0]) * 0.15, p=int(digits[1]) / 20.0, t=int(digits[3:]) / 100.0)
    raise ValueError(f"unknown NACA designation {name!r}")


def naca_dense_contour(name, n_pts, chord, x0, y0):
    """Dense closed contour: upper surface LE->TE then lower TE->LE, cosine
    spacing in x, thickness applied normal to the camber line."""
    spec = naca_spec(name)
    beta = np.linspace(0.0, np.pi, n_pts)
    xc = 0.5 * (1.0 - np.cos(beta))
    yt = naca_thickness(xc, spec['t'])
    if spec['kind'] == 'naca4':
        yc, dyc = naca4_camber(xc, spec['m'], spec['p'])
    else:
        yc, dyc = naca5_camber(xc, spec['cli'], spec['p'])
    th = np.arctan(dyc)
    upper = np.column_stack([(xc - yt * np.sin(th)) * chord + x0, (yc + yt * np.cos(th)) * chord + y0])
    lower = np.column_stack([(xc + yt * np.sin(th)) * chord + x0, (yc - yt * np.cos(th)) * chord + y0])[::-1]
    dense = np.concatenate([upper, lower[1:-1]])
    ymid = float(np.interp(0.5, xc, yc))
    return dense, spec['t'] * chord, (x0 + 0.5 * chord, y0 + ymid * chord)


def sample_airfoil(dense, n_half, chord, x0, y0, h):
    """Body points: upper surface, trailing-edge point, lower surface
    (``mesh_utils.py:96-111``)."""
    h_body = h * 2.0 / 3.0
    h_min = h / 5.0
    upper = dense[:n_half]
    lower = np.concatenate([dense[:1], dense[n_half:][::-1], dense[n_half - 1:n_half]])
    up = sample_half_contour(upper, h_body, h_min)
    lo = sample_half_contour(lower, h_body, h_min)
    te = np.array([[x0 + chord, y0]])
    if len(up) > 1 and np.linalg.norm(up[-1] - te[0]) < 0.5 * h_body:
        up = up[:-1]
    if len(lo) > 1 and np.linalg.norm(lo[-1] - te[0]) < 0.5 * h_body:
        lo = lo[:-1]
    return np.concatenate([up, te, lo[::-1][:-1]])


def airfoil_size_fn(dense, cx, chord, t_max, h, sp: SizeParams = AIRFOIL_SIZE):
    """Vectorised local target size around an airfoil (``mesh_utils.py:114-141``)."""
    tree = cKDTree(dense)
    kappa = menger_curvature(dense)
    x_le = cx - chord / 2.0
    growth_length = max(t_max, h)

    def fn(pts):
        pts = np.atleast_2d(np.asarray(pts, float))
        dist, idx = tree.query(pts)
        k = np.maximum(kappa[idx], 1e-10)
        h_surf = np.clip(h / k, h / 5.0, h * 2.0 / 3.0)
        h_base = h_surf + np.minimum(1.0, dist / h) * (h - h_surf)
        gap = x_le - pts[:, 0]
        blend = smoothstep(gap / max(sp.left_margin_factor * t_max, 4.0 * h))
        gr = sp.growth_rate + blend * (sp.left_growth_rate - sp.growth_rate)
        msf = sp.max_size_factor * (1.0 + 3.0 * blend)
        target = h_base * (1.0 + gr * dist / growth_length)
        out = np.clip(target, h_base, msf * h)
        out = np.where(dist <= sp.obstacle_factor * t_max, h, out)
        return out
    return fn


# --------------------------------------------------------------------------
# Diamond
# --------------------------------------------------------------------------

def diamond_vertices(cx, cy, chord, height):
    hc, ht = chord / 2.0, height / 2.0
    return np.array([(cx - hc, cy), (cx, cy + ht), (cx + hc, cy), (cx, cy - ht)])


def sample_loop(verts, h):
    """ceil(len/h) (at least 2) uniform points per side, endpoint excluded."""
    pts = []
    for i in range(len(verts)):
        p0, p1 = verts[i], verts[(i + 1) % len(verts)]
        n = max(2, int(np.ceil(np.linalg.norm(p1 - p0) / h)))
        pts.append(np.linspace(p0, p1, n, endpoint=False))
    return np.concatenate(pts)


def diamond_distance(pts, cx, cy, chord, height):
    """Distance to the rhombus |x'|+|y'| <= 1 measured as the reference does:
    to the radial projection on the rhombus boundary (``diamond.py:32-40``)."""
    pts = np.atleast_2d(np.asarray(pts, float))
    px = (pts[:, 0] - cx) / (chord / 2.0)
    py = (pts[:, 1] - cy) / (height / 2.0)
    s = np.abs(px) + np.abs(py)
    inside = s <= 1.0
    s = np.where(s == 0, 1.0, s)
    near = np.column_stack([cx + np.sign(px) * (np.abs(px) / s) * (chord / 2.0),
                            cy + np.sign(py) * (np.abs(py) / s) * (height / 2.0)])
    d = np.linalg.norm(pts - near, axis=1)
    return np.where(inside, 0.0, d)


def diamond_size_fn(cx, cy, chord, height, h, sp: SizeParams = DIAMOND_SIZE):
    """Vectorised ``diamond.py:43-60``."""
    x_le = cx - chord / 2.0
    growth_length = max(height, h)

    def fn(pts):
        pts = np.atleast_2d(np.asarray(pts, float))
        dist = diamond_distance(pts, cx, cy, chord, height)
        gap = x_le - pts[:, 0]
        blend = smoothstep(gap / max(sp.left_margin_factor * height, 4.0 * h))
        gr = sp.growth_rate + blend * (sp.left_growth_rate - sp.growth_rate)
        msf = sp.max_size_factor * (1.0 + 3.0 * blend)
        target = h * (1.0 + gr * dist / growth_length)
        out = np.clip(target, h, msf * h)
        return np.where(dist <= sp.obstacle_factor * height, h, out)
    return fn


def box_boundary(box, size_fn, h):
    """Outer box sampled side by side: bottom, right, top, left (the left one
    is the inlet)."""
    x0, x1, y0, y1 = box
    corners = [(x0, y0), (x1, y0), (x1, y1), (x0, y1)]
    pts, last = [], None
    scalar = lambda p: float(size_fn(np.asarray(p)[None])[0])
    for i in range(4):
        seg = sample_segment(corners[i], corners[(i + 1) % 4], scalar, min_step=h)
        if last is not None and len(seg) and np.allclose(seg[0], last):
            seg = seg[1:]
        pts.append(seg)
        if len(seg):
            last = seg[-1]
    return np.concatenate(pts)
