"""ctypes wrapper of the C/OpenMP restatement of the oracle (oracle/cport/esr_cpu.c).

TEST INFRASTRUCTURE ONLY: the multi-threaded CPU baseline and a cross-check
of the NumPy oracle. ``make -C oracle`` builds ``oracle/libesr_cpu.so``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from . import euler_oracle as O

HERE = Path(__file__).resolve().parent
LIB = HERE / "libesr_cpu.so"
_lib = None


def build():
    src = HERE / "cport" / "esr_cpu.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
    return _lib


class CpuCase:
    """Geometry of one mesh laid out for the C step, from the oracle's own
    geometry formulas, plus the freestream and sponge of one case."""

    def __init__(self, mesh, mach, aoa, dtype=np.float64, gamma=1.4):
        self.dtype = dtype
        om = O.build_oracle_mesh(mesh.points, mesh.tris, mesh.neighbors, mesh.faces, mesh.face_markers,
                                 mesh.face_connectivity, dtype=dtype, metadata=mesh.metadata)
        self.om = om
        n = mesh.n_cells
        mk = mesh.face_markers[mesh.face_connectivity]
        wall = set(mesh.metadata.get('wall_markers', [2]))
        kind = np.where(mk == 0, 0, np.where(mk == 3, 3, np.where(mk == 4, 4, np.where(np.isin(mk, list(wall)), 2, 4))))
        self.nbr = np.ascontiguousarray(np.where(mesh.neighbors >= 0, mesh.neighbors, 0), dtype=np.int32)
        self.kind = np.ascontiguousarray(kind, dtype=np.int32)
        mid = O.face_midpoints(om)
        bary = om.barycenter
        dxf = mid - bary[:, None, :]
        dxl = np.where((mk > 0)[..., None], dtype(2) * dxf, bary[self.nbr] - bary[:, None, :])
        dxn = mid - bary[self.nbr]
        self.nrm = np.ascontiguousarray(om.normals, dtype=dtype)
        self.s = np.ascontiguousarray(om.surface[mesh.face_connectivity], dtype=dtype)
        self.dxf = np.ascontiguousarray(dxf, dtype=dtype)
        self.dxl = np.ascontiguousarray(dxl, dtype=dtype)
        self.dxn = np.ascontiguousarray(dxn, dtype=dtype)
        self.area = np.ascontiguousarray(om.area, dtype=dtype)
        cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=gamma, Mach=mach, aoa=aoa, case=mesh.metadata.get('case', 'diamond'))
        W, inlet = O.initialize(n, cfg, dtype)
        self.W0, self.inlet = W, inlet
        # sponge coefficient sigma_c = strength * blend^3 (helper.py:262-295): the
        # sponge source at W = 0 is sigma * inlet, and the inlet density is rho_inf
        probe = O.sponge_source(np.zeros_like(W), om, inlet, gamma)
        self.sigma = np.ascontiguousarray(probe[:, 0] / inlet[0], dtype=dtype)
        self.gamma = gamma
        self.dt = O.get_dt(W, om, CFL=0.45 if (0.6 < mach < 1.1) else 0.6, gamma=gamma)

    def srk2(self, W, nsteps):
        W = np.ascontiguousarray(W, dtype=self.dtype).copy()
        L = lib()
        f = L.esr_cpu_srk2_f64 if self.dtype == np.float64 else L.esr_cpu_srk2_f32
        ct = C.c_double if self.dtype == np.float64 else C.c_float
        p = lambda a, t=ct: a.ctypes.data_as(C.POINTER(t))
        n = self.area.shape[0]
        inl = np.ascontiguousarray(self.inlet, dtype=self.dtype)
        rc = f(n, p(self.nbr, C.c_int32), p(self.kind, C.c_int32), p(self.nrm), p(self.s), p(self.dxf), p(self.dxl),
               p(self.dxn), p(self.area), p(self.sigma), ct(self.gamma), p(inl), ct(self.dt), int(nsteps), p(W))
        if rc != 0:
            raise MemoryError("esr_cpu_srk2: allocation failed")
        return W

    def srk2_local(self, W, nsteps, cfl):
        """nsteps SRK2 steps with the per-cell CFL step (oracle time_step_srk2_local)."""
        W = np.ascontiguousarray(W, dtype=self.dtype).copy()
        L = lib()
        f = L.esr_cpu_srk2_local_f64 if self.dtype == np.float64 else L.esr_cpu_srk2_local_f32
        ct = C.c_double if self.dtype == np.float64 else C.c_float
        p = lambda a, t=ct: a.ctypes.data_as(C.POINTER(t))
        n = self.area.shape[0]
        inl = np.ascontiguousarray(self.inlet, dtype=self.dtype)
        rc = f(n, p(self.nbr, C.c_int32), p(self.kind, C.c_int32), p(self.nrm), p(self.s), p(self.dxf), p(self.dxl),
               p(self.dxn), p(self.area), p(self.sigma), ct(self.gamma), p(inl), ct(cfl), int(nsteps), p(W))
        if rc != 0:
            raise MemoryError("esr_cpu_srk2_local: allocation failed")
        return W


def threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
