"""Quality triangular meshes of a box with one body cut out.

The reference meshes with Triangle through meshpy (a constrained Delaunay
triangulation refined until every triangle is under the size function's area
and above 30 degrees, ``euler/meshing/mesh_utils.py:182-198``); neither is
available here, so this module is a new mesher on top of SciPy's Delaunay:

1. the outer box and the body contour are sampled into boundary segments;
2. segments whose diametral circle holds another point ("encroached") are
   split until none is, so every segment is a Delaunay edge and the
   unconstrained Delaunay triangulation conforms to the boundary. Segments
   touching a sharp body vertex (interior angle < 60 degrees, e.g. the diamond
   and trailing-edge tips) are split on concentric shells, at distances
   h * 2^k from the tip, so the two sides of the tip never encroach each
   other without end;
3. Delaunay refinement in batches: triangles larger than the size-function
   area or with an angle under ``min_angle`` get their circumcentre inserted,
   unless it would encroach a segment, in which case that segment is split
   instead; circumcentres too close to one another in the same batch are
   thinned out;
4. triangles inside the body are dropped; the result is oriented CCW and
   converted to the solver's connectivity with box-side boundary markers.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.spatial import Delaunay, cKDTree

from ..mesh import Mesh, classify_box_markers, WALL
from . import contours as C


# Batch insertion lands closer to the area bound than Triangle's one-at-a-time
# insertion; this factor on the bound brings the cell counts of the reference
# meshes (diamond ~1.4k cells at h=0.1, ~20.2k at h=0.025) back.
AREA_SCALE = 1.2


def points_in_polygon(pts, poly):
    """Even-odd ray casting, vectorised over points."""
    pts = np.asarray(pts, float)
    x, y = pts[:, 0][:, None], pts[:, 1][:, None]
    xa, ya = poly[:, 0][None, :], poly[:, 1][None, :]
    xb, yb = np.roll(poly[:, 0], -1)[None, :], np.roll(poly[:, 1], -1)[None, :]
    out = np.zeros(len(pts), dtype=bool)
    step = 20000
    for s in range(0, len(pts), step):
        xs, ys = x[s:s + step], y[s:s + step]
        cond = (ya > ys) != (yb > ys)
        with np.errstate(divide='ignore', invalid='ignore'):
            xint = xa + (ys - ya) * (xb - xa) / (yb - ya)
        crossing = cond & (xs < xint)
        out[s:s + step] = (np.count_nonzero(crossing, axis=1) % 2) == 1
    return out


def _interior_angles(poly):
    """Interior angle (degrees) at each vertex of a CCW polygon."""
    prev = np.roll(poly, 1, axis=0)
    nxt = np.roll(poly, -1, axis=0)
    a = prev - poly
    b = nxt - poly
    ang_a = np.arctan2(a[:, 1], a[:, 0])
    ang_b = np.arctan2(b[:, 1], b[:, 0])
    # CCW polygon: interior lies to the left walking prev -> v -> next
    d = np.degrees((ang_a - ang_b) % (2 * np.pi))
    return d


class _Segments:
    """Boundary segments as index pairs with a 'sharp tip' flag per end."""

    def __init__(self):
        self.a, self.b, self.ta, self.tb = [], [], [], []

    def add_loop(self, start, n, tips=None):
        for i in range(n):
            j = (i + 1) % n
            self.a.append(start + i)
            self.b.append(start + j)
            self.ta.append(bool(tips is not None and tips[i]))
            self.tb.append(bool(tips is not None and tips[j]))

    def arrays(self):
        return np.asarray(self.a), np.asarray(self.b)


def _split_point(pa, pb, tip_a, tip_b, unit):
    """Midpoint, or the concentric-shell point nearest the midpoint when one end
    is a sharp tip."""
    L = float(np.linalg.norm(pb - pa))
    if tip_a == tip_b:
        return 0.5 * (pa + pb)
    k = math.floor(math.log2(0.5 * L / unit) + 0.5)
    d = unit * 2.0 ** k
    if not (0.25 * L <= d <= 0.75 * L):
        d = 0.5 * L
    if tip_a:
        return pa + (pb - pa) * (d / L)
    return pb + (pa - pb) * (d / L)


def refine(outer, body, size_fn, h, min_angle=30.0, max_rounds=400, tip_angle=60.0, area_scale=AREA_SCALE):
    """Mesh the box polygon ``outer`` (CCW, sampled) minus the body polygon
    ``body`` (CCW, sampled). Returns (points, CCW triangles)."""
    outer = np.asarray(outer, float)
    body = np.asarray(body, float)
    body_ccw = body if _signed_area(body) > 0 else body[::-1]
    tips = _interior_angles(body_ccw) < tip_angle
    pts = [p for p in outer] + [p for p in body_ccw]
    segs = _Segments()
    segs.add_loop(0, len(outer))
    segs.add_loop(len(outer), len(body_ccw), tips)
    unit = h
    bmin = outer.min(0)
    bmax = outer.max(0)
    sin_min = math.sin(math.radians(min_angle))
    P = np.asarray(pts)

    def split_segments(idx_list):
        nonlocal P
        new_pts = []
        for s in sorted(set(idx_list), reverse=True):
            a, b = segs.a[s], segs.b[s]
            p = _split_point(P[a], P[b], segs.ta[s], segs.tb[s], unit)
            k = len(P) + len(new_pts)
            new_pts.append(p)
            tb = segs.tb[s]
            segs.b[s] = k
            segs.tb[s] = False
            segs.a.append(k); segs.b.append(b); segs.ta.append(False); segs.tb.append(tb)
        if new_pts:
            P = np.vstack([P, np.asarray(new_pts)])

    for _ in range(max_rounds):
        # (2) remove all segment encroachment
        for _inner in range(200):
            A, B = segs.arrays()
            mid = 0.5 * (P[A] + P[B])
            rad = 0.5 * np.linalg.norm(P[B] - P[A], axis=1)
            tree = cKDTree(P)
            hits = tree.query_ball_point(mid, rad * (1 - 1e-9))
            enc = [s for s, lst in enumerate(hits) if any((q != A[s] and q != B[s]) for q in lst)]
            if not enc:
                break
            split_segments(enc)
        # (3) quality refinement
        tri = Delaunay(P)
        T = tri.simplices
        cen = P[T].mean(axis=1)
        keep = ~points_in_polygon(cen, body_ccw)
        T = T[keep]
        X = P[T]
        e0 = X[:, 1] - X[:, 0]
        e1 = X[:, 2] - X[:, 1]
        e2 = X[:, 0] - X[:, 2]
        l0, l1, l2 = (np.linalg.norm(e, axis=1) for e in (e0, e1, e2))
        area = 0.5 * np.abs(e0[:, 0] * (-e2[:, 1]) - e0[:, 1] * (-e2[:, 0]))
        R = l0 * l1 * l2 / np.maximum(4 * area, 1e-300)
        lmin = np.minimum(np.minimum(l0, l1), l2)
        target = area_scale * C.triangle_area_from_h(size_fn(cen[keep]))
        too_big = area > target
        skinny = (R / np.maximum(lmin, 1e-300)) > 1.0 / (2 * sin_min) * (1 + 1e-9)
        # triangles squeezed between two segments at a sharp tip cannot be fixed
        bad = too_big | (skinny & (lmin > 1e-3 * h))
        if not np.any(bad):
            break
        Xb = X[bad]
        ax, ay = Xb[:, 0, 0], Xb[:, 0, 1]
        bx, by = Xb[:, 1, 0], Xb[:, 1, 1]
        cx, cy = Xb[:, 2, 0], Xb[:, 2, 1]
        d = 2 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by))
        ux = ((ax ** 2 + ay ** 2) * (by - cy) + (bx ** 2 + by ** 2) * (cy - ay) + (cx ** 2 + cy ** 2) * (ay - by)) / d
        uy = ((ax ** 2 + ay ** 2) * (cx - bx) + (bx ** 2 + by ** 2) * (ax - cx) + (cx ** 2 + cy ** 2) * (bx - ax)) / d
        cc = np.column_stack([ux, uy])
        Rb = R[bad]
        prio = np.argsort(-(area[bad] / target[bad]))
        cc, Rb = cc[prio], Rb[prio]
        A, B = segs.arrays()
        mid = 0.5 * (P[A] + P[B])
        rad = 0.5 * np.linalg.norm(P[B] - P[A], axis=1)
        stree = cKDTree(mid)
        rmax = float(rad.max())
        near = stree.query_ball_point(cc, rmax)
        to_split = set()
        accepted = []
        acc_tree_pts = []
        for i in range(len(cc)):
            p = cc[i]
            enc = [s for s in near[i] if np.linalg.norm(p - mid[s]) < rad[s]]
            if enc:
                to_split.update(enc)
                continue
            if not (bmin[0] < p[0] < bmax[0] and bmin[1] < p[1] < bmax[1]):
                continue
            if acc_tree_pts:
                dd = np.min(np.linalg.norm(np.asarray(acc_tree_pts) - p, axis=1))
                if dd < 0.5 * Rb[i]:
                    continue
            accepted.append(p)
            acc_tree_pts.append(p)
            if len(acc_tree_pts) > 4000:
                break
        if accepted:
            acc = np.asarray(accepted)
            inside_body = points_in_polygon(acc, body_ccw)
            acc = acc[~inside_body]
            P = np.vstack([P, acc])
        if to_split:
            split_segments(list(to_split))
        if not accepted and not to_split:
            break
    tri = Delaunay(P)
    T = tri.simplices
    keep = ~points_in_polygon(P[T].mean(axis=1), body_ccw)
    T = T[keep]
    # drop unused points, keep order
    used = np.zeros(len(P), bool)
    used[T.reshape(-1)] = True
    remap = -np.ones(len(P), dtype=np.int64)
    remap[used] = np.arange(used.sum())
    return P[used], remap[T]


def _signed_area(poly):
    x, y = poly[:, 0], poly[:, 1]
    return 0.5 * float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


def _finish(points, tris, box, metadata, renumber=True) -> Mesh:
    mesh = Mesh.from_triangles(points, tris, markers=lambda p, f, b: classify_box_markers(p, f, b, box),
                               metadata=metadata)
    if renumber:
        mesh = mesh.renumbered(mesh.rcm_permutation())
    mesh.validate()
    return mesh


def diamond_mesh(h=0.1, Lx=4.0, Ly=4.0, chord=1.0, half_angle_deg=5.0, cx=1.5, cy=2.0,
                 case='diamond', min_angle=30.0, renumber=True) -> Mesh:
    """Diamond (rhombus) airfoil in [0,Lx]x[0,Ly]; the reference's defaults:
    chord 1 at (1.5, 2), height = chord * tan(half angle)
    (``euler/generate_mesh.py:28-32``, ``euler/meshing/diamond.py:82-108``)."""
    height = chord * math.tan(math.radians(half_angle_deg))
    verts = C.diamond_vertices(cx, cy, chord, height)
    box = (0.0, Lx, 0.0, Ly)
    size = C.diamond_size_fn(cx, cy, chord, height, h)
    outer = C.box_boundary(box, size, h)
    body = C.sample_loop(verts, h)
    pts, tris = refine(outer, body, size, h, min_angle=min_angle)
    md = dict(case=case, h=h, domain={"Lx": Lx, "Ly": Ly}, obstacle_length=chord, chord=chord,
              height=height, center={"cx": cx, "cy": cy}, symmetric=False, wall_markers=[WALL],
              force_marker=WALL, mesher="eulersr_b200.meshing")
    return _finish(pts, tris, box, md, renumber)


def airfoil_mesh(name='naca0012', h=0.1, Lx=4.0, Ly=4.0, chord=1.0, cx=1.5, cy=2.0,
                 min_angle=30.0, renumber=True) -> Mesh:
    """NACA 4- or 5-digit airfoil from its analytic formulas in [0,Lx]x[0,Ly],
    chord 1 with the leading edge at cx - chord/2 (``euler/generate_mesh.py:18``)."""
    x_le = cx - chord / 2.0
    dense, t_max, _hole = C.naca_dense_contour(name, 2000, chord, x_le, cy)
    box = (0.0, Lx, 0.0, Ly)
    size = C.airfoil_size_fn(dense, cx, chord, t_max, h)
    outer = C.box_boundary(box, size, h)
    body = C.sample_airfoil(dense, 2000, chord, x_le, cy, h)
    pts, tris = refine(outer, body, size, h, min_angle=min_angle)
    spec = C.naca_spec(name)
    md = dict(case=name.lower(), h=h, domain={"Lx": Lx, "Ly": Ly}, obstacle_length=chord, chord=chord,
              thickness=spec['t'], height=t_max, center={"cx": cx, "cy": cy}, wall_markers=[WALL],
              force_marker=WALL, mesher="eulersr_b200.meshing")
    return _finish(pts, tris, box, md, renumber)


def build_mesh(geometry: str, h: float, **kw) -> Mesh:
    g = geometry.lower()
    if g.startswith('diamond'):
        return diamond_mesh(h=h, case=g, **kw)
    if g.startswith('naca'):
        return airfoil_mesh(g, h=h, **kw)
    raise ValueError(f"unknown geometry {geometry!r}")
