"""Geometry-only inputs of the warm-start model, computed once per mesh pair.

* k-nearest LR cells of every HR cell (k=6, scipy cKDTree on barycentres,
  ``eval/testset.py:309-316``): indices and distances for the IDW kernel;
* wall distance and outward wall normal of every HR cell from 8 samples per
  wall face (``utils/aero.py:154-177``);
* HR barycentres centred on the body and scaled by its chord.

Everything that depends on a case (IDW of the LR solution, the feature rows,
the MLP) runs on the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.spatial import cKDTree

from ..mesh import Mesh

MACH_MID = (0.7 + 3.0) / 2      # preprocessing/dataset.py:12-14
MACH_SCALE = (3.0 - 0.7) / 2
AOA_SCALE = 5.0


def wall_features(mesh: Mesh, query, n_samp=8):
    """Distance to the wall and the wall normal pointing towards each query
    point (utils/aero.py:154-177)."""
    wf, cells, slots = mesh.wall_owner_data()
    a = mesh.points[mesh.faces[wf, 0]]
    b = mesh.points[mesh.faces[wf, 1]]
    # body-outward normal = minus the fluid cell's outward normal
    nrm = -mesh.normals[cells, slots]
    t = np.linspace(0.0, 1.0, n_samp)[None, :, None]
    samples = (a[:, None, :] * (1 - t) + b[:, None, :] * t).reshape(-1, 2)
    d, idx = cKDTree(samples).query(np.asarray(query, np.float64))
    seg = idx // n_samp
    n = nrm[seg]
    mid = 0.5 * (a + b)
    sgn = np.sign(((np.asarray(query) - mid[seg]) * n).sum(1, keepdims=True))
    return d, n * np.where(sgn == 0, 1.0, sgn)


@dataclass
class MeshPair:
    hr: Mesh
    lr: Mesh
    knn_idx: np.ndarray       # (N_hr, 6) int32 LR cell ids
    knn_dist: np.ndarray      # (N_hr, 6) float32
    static5: np.ndarray       # (N_hr, 5) float32: x, y (centred/chord), wall distance/chord, wall normal
    center: tuple
    chord: float

    @classmethod
    def build(cls, hr: Mesh, lr: Mesh, k=6):
        chord = float(hr.metadata.get("obstacle_length", hr.metadata.get("chord", 1.0)) or 1.0)
        c = hr.metadata.get("center", {"cx": 1.5, "cy": 2.0})
        center = (float(c.get("cx", 1.5)), float(c.get("cy", 2.0)))
        d, idx = cKDTree(lr.barycenter).query(hr.barycenter, k=k)
        wd, wn = wall_features(hr, hr.barycenter)
        pos = (hr.barycenter - np.asarray(center)[None, :]) / chord
        st = np.column_stack([pos, wd / chord, wn]).astype(np.float32)
        return cls(hr, lr, idx.astype(np.int32), d.astype(np.float32), st, center, chord)
