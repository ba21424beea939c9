"""Mesh generation for the solver's test geometries (diamond, NACA 4/5-digit)."""
from .mesher import build_mesh, diamond_mesh, airfoil_mesh, refine  # noqa: F401
