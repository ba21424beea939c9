"""Unstructured triangular mesh: connectivity, geometry and file formats.

The attribute set and its conventions are those the EulerSR solver reads
(``euler/jax_fvm/src/mesh.py:28-150``), so that meshes move between the two
code bases unchanged:

* ``tris`` are counter-clockwise; edge k of a triangle joins vertex k and k+1;
* ``neighbors[c, k]`` is the cell across edge k, -1 on the boundary
  (``euler/meshing/mesh_utils.py:173-179,268-288``);
* ``face_connectivity[c, k]`` is the face id of edge k (``mesh.py:242-260``);
* ``normals[c, k]`` is the outward unit normal of edge k, (dy, -dx)/len
  (``mesh.py:226-230``);
* face markers: 0 interior, 2 wall, 3 inlet, 4 outlet, 5 subsonic inlet
  (``mesh.py:47-52``).

Geometry is always computed in float64 here; kernels round it once to their
working precision.

File formats:

* ``graph.npz`` as ``euler/graph.py:5-108`` writes it (directed edges, edge
  normals, lengths, BC markers), extended with the arrays the solver needs and
  that format lacks (``points``, ``tris``, ``faces``, ``face_markers``,
  ``face_connectivity``, ``neighbors``, ``face_mid``) plus the metadata as JSON;
* the reference's pickled ``Mesh`` ``.npy`` files (``mesh.py:327-359``), read
  through an unpickler that maps JAX arrays to NumPy without importing JAX.
"""
from __future__ import annotations

import io
import json
import pickle
import os
from pathlib import Path
from typing import Any

import numpy as np

WALL, INLET, OUTLET, SUBSONIC_INLET = 2, 3, 4, 5


def faces_neighbors_from_tris(tris: np.ndarray):
    """Unique faces, per-edge neighbours and per-edge face ids from CCW
    triangles (vectorised form of ``mesh_utils.py:268-288`` and
    ``mesh.py:242-260``). Faces are ordered by their sorted vertex pair."""
    tris = np.asarray(tris, dtype=np.int64)
    n = tris.shape[0]
    a = tris
    b = np.roll(tris, -1, axis=1)
    lo = np.minimum(a, b).reshape(-1)
    hi = np.maximum(a, b).reshape(-1)
    key = lo * (int(hi.max(initial=0)) + 1) + hi
    uniq, first, inv, counts = np.unique(key, return_index=True, return_inverse=True, return_counts=True)
    if np.any(counts > 2):
        raise ValueError("non-manifold mesh: an edge is shared by more than two triangles")
    faces = np.stack([lo[first], hi[first]], axis=1)
    face_conn = inv.reshape(n, 3)
    # pair up the two slots of each interior face
    order = np.argsort(inv, kind='stable')
    sorted_inv = inv[order]
    neighbors = -np.ones(3 * n, dtype=np.int64)
    same = sorted_inv[1:] == sorted_inv[:-1]
    s0 = order[:-1][same]
    s1 = order[1:][same]
    neighbors[s0] = s1 // 3
    neighbors[s1] = s0 // 3
    boundary = counts == 1
    return faces.astype(np.int32), neighbors.reshape(n, 3).astype(np.int32), face_conn.astype(np.int32), boundary


def classify_box_markers(points, faces, boundary, box, tol=1e-6):
    """Boundary markers by position (``mesh_utils.py:291-303``): the left side
    of the box is the inlet, the other three sides outlets, anything else a
    wall. ``box`` = (x0, x1, y0, y1)."""
    x0, x1, y0, y1 = box
    markers = np.zeros(len(faces), dtype=np.int32)
    f = np.where(boundary)[0]
    pa = points[faces[f, 0]]
    pb = points[faces[f, 1]]
    left = (pa[:, 0] < x0 + tol) & (pb[:, 0] < x0 + tol)
    right = (pa[:, 0] > x1 - tol) & (pb[:, 0] > x1 - tol)
    bottom = (pa[:, 1] < y0 + tol) & (pb[:, 1] < y0 + tol)
    top = (pa[:, 1] > y1 - tol) & (pb[:, 1] > y1 - tol)
    m = np.full(len(f), WALL, dtype=np.int32)
    m[right | bottom | top] = OUTLET
    m[left] = INLET
    markers[f] = m
    return markers


class Mesh:
    """Mesh record with the reference's attribute names (``mesh.py:32-45``)."""

    points: np.ndarray
    tris: np.ndarray
    neighbors: np.ndarray
    faces: np.ndarray
    face_markers: np.ndarray
    face_connectivity: np.ndarray
    face_connectivity_opposite: np.ndarray
    barycenter: np.ndarray
    area: np.ndarray
    surface: np.ndarray
    normals: np.ndarray
    metadata: dict

    def __init__(self, **kwargs):
        self.metadata = {}
        for k, v in kwargs.items():
            setattr(self, k, v)

    # ------------------------------------------------------------------ build
    @classmethod
    def from_arrays(cls, points, tris, neighbors, faces, face_markers, face_connectivity=None,
                    metadata: dict | None = None, face_connectivity_opposite=None) -> "Mesh":
        """Mirror of ``Mesh.mesh_generator_from_points`` (``mesh.py:131-150``)."""
        m = cls()
        m.points = np.asarray(points, dtype=np.float64)
        m.tris = np.asarray(tris, dtype=np.int32)
        m.neighbors = np.asarray(neighbors, dtype=np.int32)
        m.faces = np.asarray(faces, dtype=np.int32)
        m.face_markers = np.asarray(face_markers, dtype=np.int32)
        if face_connectivity is None:
            face_connectivity = _face_connectivity_lookup(m.faces, m.tris)
        m.face_connectivity = np.asarray(face_connectivity, dtype=np.int32)
        if face_connectivity_opposite is None:
            face_connectivity_opposite = np.arange(m.faces.shape[0], dtype=np.int32)
        m.face_connectivity_opposite = np.asarray(face_connectivity_opposite, dtype=np.int32)
        m.metadata = dict(metadata or {})
        m.compute_geometry()
        return m

    @classmethod
    def from_triangles(cls, points, tris, box=None, markers=None, metadata=None) -> "Mesh":
        """Build connectivity from CCW triangles; boundary markers come from
        ``markers`` (callable(points, faces, boundary) -> markers) or from the
        box classification."""
        points = np.asarray(points, dtype=np.float64)
        tris = np.asarray(tris, dtype=np.int64)
        P = points[tris]
        cross = (P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1]) - (P[:, 1, 1] - P[:, 0, 1]) * (P[:, 2, 0] - P[:, 0, 0])
        cw = cross < 0
        tris = tris.copy()
        tris[cw] = tris[cw][:, ::-1]
        faces, neighbors, fc, boundary = faces_neighbors_from_tris(tris)
        if markers is not None:
            fm = markers(points, faces, boundary)
        else:
            if box is None:
                box = (points[:, 0].min(), points[:, 0].max(), points[:, 1].min(), points[:, 1].max())
            fm = classify_box_markers(points, faces, boundary, box)
        return cls.from_arrays(points, tris, neighbors, faces, fm, fc, metadata)

    def compute_geometry(self):
        """``mesh.py:223-240`` in float64."""
        P = self.points[self.tris]
        self.barycenter = P.mean(axis=1)
        d = np.roll(P, -1, axis=1) - P
        ln = np.linalg.norm(d, axis=-1)
        self.normals = np.stack([d[..., 1], -d[..., 0]], -1) / ln[..., None]
        self.area = np.abs(0.5 * ((P[:, 1, 1] - P[:, 0, 1]) * (P[:, 2, 0] - P[:, 0, 0])
                                  - (P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1])))
        self.surface = np.linalg.norm(self.points[self.faces[:, 1]] - self.points[self.faces[:, 0]], axis=1)
        return self

    # --------------------------------------------------------------- queries
    @property
    def n_cells(self) -> int:
        return int(self.tris.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.faces.shape[0])

    def face_midpoints(self) -> np.ndarray:
        return self.points[self.faces].mean(axis=1)

    def wall_markers(self):
        wm = self.metadata.get('wall_markers', [WALL])
        try:
            return tuple(int(m) for m in wm)
        except TypeError:
            return (int(wm),)

    def force_marker(self) -> int:
        return int(self.metadata.get('force_marker', WALL))

    def wall_owner_data(self, marker: int | None = None):
        """Owner cell and slot of each face carrying ``marker``: the first
        (lowest index) cell listing the face, as ``helper.py:373-379`` picks it."""
        marker = self.force_marker() if marker is None else marker
        wall_faces = np.where(self.face_markers == marker)[0]
        fc = self.face_connectivity.reshape(-1)
        # first occurrence of every face id in row-major (cell, slot) order
        first = np.full(self.n_faces, -1, dtype=np.int64)
        idx = np.arange(fc.size)
        order = np.argsort(fc, kind='stable')
        fcs = fc[order]
        starts = np.r_[0, np.nonzero(np.diff(fcs))[0] + 1]
        first[fcs[starts]] = idx[order][starts]
        pos = first[wall_faces]
        return wall_faces.astype(np.int32), (pos // 3).astype(np.int32), (pos % 3).astype(np.int32)

    def quality(self) -> dict:
        P = self.points[self.tris]
        e = np.linalg.norm(np.roll(P, -1, axis=1) - P, axis=-1)
        a, b, c = e[:, 0], e[:, 1], e[:, 2]
        cosA = np.clip((b ** 2 + c ** 2 - a ** 2) / (2 * b * c), -1, 1)
        cosB = np.clip((a ** 2 + c ** 2 - b ** 2) / (2 * a * c), -1, 1)
        cosC = np.clip((a ** 2 + b ** 2 - c ** 2) / (2 * a * b), -1, 1)
        ang = np.degrees(np.arccos(np.stack([cosA, cosB, cosC], 1)))
        return {'n_cells': self.n_cells, 'n_faces': self.n_faces, 'n_points': int(self.points.shape[0]),
                'min_angle_deg': float(ang.min()), 'max_angle_deg': float(ang.max()),
                'min_area': float(self.area.min()), 'max_area': float(self.area.max())}

    def validate(self):
        """Structural checks: CCW cells, symmetric neighbours, face slots
        consistent with edges, markers zero exactly on interior faces."""
        assert np.all(self.area > 0), "degenerate cell"
        P = self.points[self.tris]
        cross = (P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1]) - (P[:, 1, 1] - P[:, 0, 1]) * (P[:, 2, 0] - P[:, 0, 0])
        assert np.all(cross > 0), "cells must be counter-clockwise"
        n = self.neighbors
        c, k = np.nonzero(n >= 0)
        nb = n[c, k]
        assert np.all(np.any(self.neighbors[nb] == c[:, None], axis=1)), "neighbours not symmetric"
        assert np.all(self.face_connectivity[c, k][:, None] == self.face_connectivity[nb][
            np.arange(len(nb))[:, None], np.argmax(self.neighbors[nb] == c[:, None], axis=1)[:, None]]), \
            "shared face ids differ"
        bnd = n < 0
        assert np.all(self.face_markers[self.face_connectivity[bnd]] > 0), "boundary face without marker"
        assert np.all(self.face_markers[self.face_connectivity[~bnd]] == 0), "interior face with marker"
        return True

    # ------------------------------------------------------------- renumber
    def rcm_permutation(self) -> np.ndarray:
        """Reverse Cuthill-McKee order of the cell adjacency graph. ``perm[i]``
        is the old index of new cell i."""
        from scipy.sparse import csr_matrix
        from scipy.sparse.csgraph import reverse_cuthill_mckee
        n = self.n_cells
        c, k = np.nonzero(self.neighbors >= 0)
        A = csr_matrix((np.ones(len(c)), (c, self.neighbors[c, k])), shape=(n, n))
        return np.asarray(reverse_cuthill_mckee(A, symmetric_mode=True), dtype=np.int64)

    def renumbered(self, perm: np.ndarray) -> "Mesh":
        """Copy with cells reordered (new cell i = old cell perm[i]); faces and
        points keep their ids."""
        perm = np.asarray(perm, dtype=np.int64)
        inv = np.empty_like(perm)
        inv[perm] = np.arange(len(perm))
        nb = self.neighbors[perm]
        nb = np.where(nb >= 0, inv[np.maximum(nb, 0)], -1)
        return Mesh.from_arrays(self.points, self.tris[perm], nb, self.faces, self.face_markers,
                                self.face_connectivity[perm], dict(self.metadata),
                                self.face_connectivity_opposite)

    # ------------------------------------------------------------------- I/O
    def graph_arrays(self, W_snapshots: dict | None = None, inlet_state=None) -> dict:
        """The arrays of ``euler/graph.py:5-108`` plus the extension keys."""
        N = self.n_cells
        nb = self.neighbors
        fc = self.face_connectivity
        src, dst, en, el, ev, ef, eb, ek = [], [], [], [], [], [], [], []
        seen = set()
        for i in range(N):
            for k in range(3):
                j = int(nb[i, k])
                f = int(fc[i, k])
                if j < 0 or j >= N:
                    src.append(i); dst.append(i); en.append(self.normals[i, k]); el.append(self.surface[f])
                    ev.append((0.0, 0.0)); ef.append(f); eb.append(int(self.face_markers[f])); ek.append(1)
                    continue
                if (i, j) in seen:
                    continue
                seen.add((i, j)); seen.add((j, i))
                v = self.barycenter[j] - self.barycenter[i]
                src += [i, j]; dst += [j, i]
                en += [self.normals[i, k], -self.normals[i, k]]
                el += [self.surface[f]] * 2
                ev += [v, -v]
                ef += [f, f]; eb += [0, 0]; ek += [0, 0]
        bc_mask = self.face_markers != 0
        arrays = dict(
            node_pos=self.barycenter.astype(np.float32),
            node_area=self.area.astype(np.float32),
            edge_index=np.array([src, dst], dtype=np.int32),
            edge_normals=np.array(en, dtype=np.float32).reshape(-1, 2),
            edge_lengths=np.array(el, dtype=np.float32),
            edge_vectors=np.array(ev, dtype=np.float32).reshape(-1, 2),
            edge_face_index=np.array(ef, dtype=np.int32),
            edge_bc_marker=np.array(eb, dtype=np.int32),
            edge_kind=np.array(ek, dtype=np.int8),
            bc_face_index=np.where(bc_mask)[0].astype(np.int32),
            bc_markers=self.face_markers[bc_mask].astype(np.int32),
            inlet_state=np.array(inlet_state if inlet_state is not None else [1.0, 1.0, 0.0, 1.0], dtype=np.float32),
            # extension: what the solver needs and graph.py does not store
            points=self.points.astype(np.float64),
            tris=self.tris.astype(np.int32),
            faces=self.faces.astype(np.int32),
            face_markers=self.face_markers.astype(np.int32),
            face_connectivity=self.face_connectivity.astype(np.int32),
            face_connectivity_opposite=self.face_connectivity_opposite.astype(np.int32),
            neighbors=self.neighbors.astype(np.int32),
            face_mid=self.face_midpoints().astype(np.float64),
            metadata_json=np.array(json.dumps(_jsonable(self.metadata))),
        )
        for t, W in (W_snapshots or {}).items():
            arrays[f"t_{t:.4f}".replace(".", "_")] = np.asarray(W, dtype=np.float32)
        return arrays

    def save(self, path, W_snapshots=None, inlet_state=None):
        """Write the extended ``graph.npz``."""
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        # write aside and rename: several processes may cache the same mesh at once
        tmp = path.with_name(f".{path.stem}.{os.getpid()}.tmp.npz")
        np.savez_compressed(tmp, **self.graph_arrays(W_snapshots, inlet_state))
        os.replace(tmp, path)
        return path

    @classmethod
    def load(cls, path) -> "Mesh":
        """Read an extended ``graph.npz`` or a reference pickled ``.npy`` mesh."""
        path = Path(path)
        if path.suffix == '.npy':
            return load_reference_pickle(path)
        with np.load(path, allow_pickle=False) as d:
            if 'tris' not in d.files:
                raise ValueError(f"{path}: plain graph.npz lacks points/tris/faces; "
                                 "the solver needs the extended format")
            md = json.loads(str(d['metadata_json'])) if 'metadata_json' in d.files else {}
            fco = d['face_connectivity_opposite'] if 'face_connectivity_opposite' in d.files else None
            return cls.from_arrays(d['points'], d['tris'], d['neighbors'], d['faces'], d['face_markers'],
                                   d['face_connectivity'], md, fco)


def _face_connectivity_lookup(faces, tris):
    """Face id of every triangle edge via a sorted-pair lookup (``mesh.py:242-260``)."""
    faces = np.asarray(faces, dtype=np.int64)
    tris = np.asarray(tris, dtype=np.int64)
    base = int(max(faces.max(initial=0), tris.max(initial=0))) + 1
    fk = np.minimum(faces[:, 0], faces[:, 1]) * base + np.maximum(faces[:, 0], faces[:, 1])
    order = np.argsort(fk)
    a = tris
    b = np.roll(tris, -1, axis=1)
    ek = np.minimum(a, b) * base + np.maximum(a, b)
    pos = np.searchsorted(fk[order], ek)
    pos = np.clip(pos, 0, len(order) - 1)
    if not np.all(fk[order][pos] == ek):
        raise ValueError("a triangle edge has no face entry")
    return order[pos].astype(np.int32)


def _jsonable(obj):
    if isinstance(obj, dict):
        return {str(k): _jsonable(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_jsonable(v) for v in obj]
    if isinstance(obj, np.generic):
        return obj.item()
    if isinstance(obj, np.ndarray):
        return obj.tolist()
    return obj


# --------------------------------------------------------------------------
# Reference pickle reader (no JAX needed)
# --------------------------------------------------------------------------

class _PickledMesh:
    """Stand-in for ``jax_fvm.src.mesh.Mesh`` during unpickling."""

    def __setstate__(self, state):
        self.__dict__.update(state)


def _reconstruct_jax_array(fun, args, arr_state, aval_state=None):
    """Replacement for JAX's array reconstructor: rebuild the NumPy value the
    pickle carries and stop there (no device put)."""
    value = fun(*args)
    value.__setstate__(arr_state)
    return value


class _ReferenceUnpickler(pickle.Unpickler):
    def find_class(self, module: str, name: str) -> Any:
        if module.startswith('jax_fvm') and name == 'Mesh':
            return _PickledMesh
        if module.startswith('jax') and name in ('_reconstruct_array', 'reconstruct_array'):
            return _reconstruct_jax_array
        if module.startswith('jax'):
            raise pickle.UnpicklingError(f"unsupported JAX object in mesh pickle: {module}.{name}")
        return super().find_class(module, name)


def load_reference_pickle(path) -> Mesh:
    """Load a reference ``Mesh`` saved with ``jnp.save`` (a pickled object in
    a 0-d object ``.npy``, ``mesh.py:327-344``), applying the same legacy
    metadata fix-ups as ``mesh.py:348-357``."""
    raw = Path(path).read_bytes()
    buf = io.BytesIO(raw)
    version = np.lib.format.read_magic(buf)
    if version == (1, 0):
        np.lib.format.read_array_header_1_0(buf, max_header_size=1 << 20)
    elif version == (2, 0):
        np.lib.format.read_array_header_2_0(buf, max_header_size=1 << 20)
    else:
        np.lib.format._read_array_header(buf, version, max_header_size=1 << 20)
    obj = _ReferenceUnpickler(buf).load()
    if isinstance(obj, np.ndarray):
        obj = obj.item()
    d = dict(obj.__dict__)
    md = dict(d.get('metadata') or {})
    for key in ("h", "Lx", "Ly", "obstacle_length", "chord", "height", "cx", "cy"):
        if key not in md and key in d:
            md[key] = d[key]
    if "obstacle_length" not in md and "chord" in d:
        md["obstacle_length"] = d["chord"]
    return Mesh.from_arrays(np.asarray(d['points']), np.asarray(d['tris']), np.asarray(d['neighbors']),
                            np.asarray(d['faces']), np.asarray(d['face_markers']),
                            np.asarray(d['face_connectivity']) if 'face_connectivity' in d else None,
                            md, np.asarray(d['face_connectivity_opposite']) if 'face_connectivity_opposite' in d else None)
