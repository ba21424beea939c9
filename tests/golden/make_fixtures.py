"""Regenerate the mesh and oracle fixtures under tests/golden/.

    python tests/golden/make_fixtures.py

Meshes come from the project's mesher (deterministic); the oracle vectors are
the NumPy restatement's float64 state after a fixed number of SRK2 steps, kept
as a regression pin of the oracle itself (the reference cannot run here).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from eulersr_b200.meshing import build_mesh  # noqa: E402
from oracle import euler_oracle as O  # noqa: E402

MESHES = [("diamond", 0.2), ("naca0012", 0.2), ("diamond", 0.1)]
PIN_STEPS = 20


def mesh_path(geom, h):
    return HERE / f"{geom}_h{h}.npz"


def oracle_pin(mesh, mach, aoa, steps, dtype=np.float64):
    om = O.build_oracle_mesh(mesh.points, mesh.tris, mesh.neighbors, mesh.faces, mesh.face_markers,
                             mesh.face_connectivity, dtype=dtype, metadata=mesh.metadata)
    cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=mach, aoa=aoa, case=mesh.metadata['case'])
    W, inlet = O.initialize(mesh.n_cells, cfg, dtype)
    dt = O.get_dt(W, om, CFL=0.6)
    for _ in range(steps):
        W = O.time_step_srk2(W, om, dt, inlet)
    return W, float(dt)


def main():
    for g, h in MESHES:
        m = build_mesh(g, h)
        m.save(mesh_path(g, h))
        print(g, h, m.n_cells)
    from eulersr_b200.mesh import Mesh
    m = Mesh.load(mesh_path("diamond", 0.2))
    W, dt = oracle_pin(m, 2.5, 5.0, PIN_STEPS)
    np.savez_compressed(HERE / "oracle_diamond_h0.2_M2.5_a5_srk2x20.npz", W=W, dt=dt, steps=PIN_STEPS)


if __name__ == "__main__":
    main()
