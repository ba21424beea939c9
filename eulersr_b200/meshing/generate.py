"""Drop-in for EulerSR's ``euler/generate_mesh.py``: the same command line
(``--geom``, ``-h/--mesh-size``, ``--out-dir``, ``--fig-dir``) over this
package's mesher.

    python -m eulersr_b200.meshing.generate                          # every geometry, default sizes
    python -m eulersr_b200.meshing.generate --geom naca2412 -h 0.1 0.05

Geometries, with the reference's boxes and placements
(``euler/generate_mesh.py:18-74``): the diamond family (``diamond``,
``diamond_tx``, ``diamond_txy``, ``diamond_alpha10``, ``diamond_big``) and the
NACA airfoils ``naca0012``, ``naca2412`` and ``naca23012``, the last from its
analytic 5-digit formula where the reference reads a ``.dat`` file. Not
built: ``bump``, ``cylinder``, the ``.dat`` airfoils (``rae2822``,
``rae2822_txy``, ``oneraD``, ``oa209``) and ``diamond_sym`` (mirrored
triangulation); the solver path does not use them. The reference also draws
each mesh to ``--fig-dir``; plotting is not part of this package, so the
option is accepted and ignored.

Each mesh is written as ``<out-dir>/<geom>_h<h>.npz`` (the extended
``graph.npz`` that ``Mesh.load`` and ``--mesh-path`` read), where the
reference writes ``<geom>_h<h>.npy`` (``euler/meshing/diamond.py:111-117``).
"""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

from .mesher import airfoil_mesh, diamond_mesh

DEFAULT_H = [0.3, 0.2, 0.15, 0.1, 0.05, 0.025]      # euler/generate_mesh.py:19
AIRFOIL_BOX = dict(Lx=4.0, Ly=4.0, chord=1.0, cx=1.5, cy=2.0)   # euler/generate_mesh.py:18


def _diamond(case, Lx=4.0, Ly=4.0, half_angle_deg=5.0, cx=1.5, cy=2.0):
    return lambda h: diamond_mesh(h=h, Lx=Lx, Ly=Ly, chord=1.0, half_angle_deg=half_angle_deg, cx=cx, cy=cy,
                                  case=case)


def _airfoil(name):
    return lambda h: airfoil_mesh(name, h=h, **AIRFOIL_BOX)


# euler/generate_mesh.py:25-74 (name -> builder of one size)
GEOMS = {
    "naca0012": _airfoil("naca0012"),
    "naca2412": _airfoil("naca2412"),
    "naca23012": _airfoil("naca23012"),
    "diamond": _diamond("diamond"),
    "diamond_tx": _diamond("diamond_tx", cx=2.0),
    "diamond_txy": _diamond("diamond_txy", cx=2.0, cy=2.5),
    "diamond_alpha10": _diamond("diamond_alpha10", half_angle_deg=10.0),
    "diamond_big": _diamond("diamond_big", Lx=6.0, Ly=6.0),
}


def cache_dir() -> Path:
    """Where generated meshes are kept between runs: $EULERSR_MESH_CACHE, else
    ``.mesh_cache`` beside the package."""
    env = os.environ.get("EULERSR_MESH_CACHE")
    return Path(env) if env else Path(__file__).resolve().parents[2] / ".mesh_cache"


def cached_mesh(geom: str, h: float):
    """The mesh of ``geom`` at size h from the cache, built and stored on
    first use (any geometry ``build_mesh`` knows, with its default box)."""
    from ..mesh import Mesh
    from .mesher import build_mesh
    p = cache_dir() / f"{geom}_h{h}.npz"
    if p.exists():
        return Mesh.load(p)
    m = build_mesh(geom, h)
    m.save(p)
    return m


def mesh_path(out_dir, geom: str, h: float) -> Path:
    return Path(out_dir) / f"{geom}_h{h}.npz"


def generate(geom: str, h: float, out_dir) -> Path:
    """Build one mesh and write it; returns its path."""
    if geom not in GEOMS:
        raise ValueError(f"unknown geometry {geom!r}; available: {', '.join(GEOMS)}")
    mesh = GEOMS[geom](float(h))
    path = mesh_path(out_dir, geom, h)
    mesh.save(path)
    print(f"{geom} h={h}: {mesh.n_cells} cells")
    print(f"Mesh saved : {path}")
    return path


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(add_help=False, description=__doc__)
    parser.add_argument("--geom", nargs="*", choices=list(GEOMS), default=list(GEOMS))
    parser.add_argument("-h", "--mesh-size", dest="h", type=float, nargs="+", default=None)
    parser.add_argument("--out-dir", default=None)
    parser.add_argument("--fig-dir", default=None)
    args = parser.parse_args(sys.argv[1:] if argv is None else list(argv))
    out_dir = Path(args.out_dir) if args.out_dir else Path("data") / "meshes"
    for geom in args.geom:
        for h in (args.h if args.h is not None else DEFAULT_H):
            generate(geom, h, out_dir)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
