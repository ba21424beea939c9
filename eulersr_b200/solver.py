"""Python face of the native solver: meshes, solver handles, cases.

Every numerical step runs in ``libeulersr.so`` on the GPU; this module only
marshals arrays. There is no CPU path: if the library or a CUDA device is
missing, the constructors raise.
"""
from __future__ import annotations

import ctypes as C
import functools
import math
from dataclasses import dataclass, field

import numpy as np

from . import _ffi as F
from .mesh import Mesh


# ------------------------------------------------------------------ cases
def freestream(mach: float, aoa_deg: float = 0.0, gamma: float = 1.4, rho_inf: float = 1.0, p_inf: float = 1.0,
               dtype=np.float64):
    """Conserved freestream state (euler/main.py:28-41): primitive
    (rho, M c cos a, M c sin a, p) converted in ``dtype``."""
    return np.asarray(_freestream_values(float(mach), float(aoa_deg), float(gamma), float(rho_inf), float(p_inf),
                                         np.dtype(dtype).str), dtype=dtype)


@functools.lru_cache(maxsize=65536)
def _freestream_values(mach, aoa_deg, gamma, rho_inf, p_inf, dtype_str):
    """freestream() as a tuple of Python floats (exact copies of the values
    rounded in the dtype), cached: a batch re-submits the same cases."""
    dtype = np.dtype(dtype_str)
    c_inf = (gamma * p_inf / rho_inf) ** 0.5
    # as euler/main.py:28-41 computes it in the run's precision: the angle,
    # its cosine and sine in `dtype`; Python-float constants ((gamma - 1)
    # formed in double and rounded once)
    a = np.deg2rad(np.asarray(aoa_deg, dtype=dtype))
    prim = np.asarray([rho_inf, mach * c_inf * np.cos(a), mach * c_inf * np.sin(a), p_inf], dtype=dtype)
    rho, u, v, p = prim
    E = p / ((gamma - 1) * 1.0 ** 2) + 0.5 * rho * (u ** 2 + v ** 2)
    return tuple(float(x) for x in np.asarray([rho, rho * u, rho * v, E], dtype=dtype))


def clamp_cfl(mach: float, cfl: float) -> float:
    """Transonic CFL clamp of euler/main.py:117-120."""
    return 0.45 if (0.6 < mach < 1.1 and cfl > 0.45) else cfl


@dataclass
class FlowCase:
    """One (Mach, alpha) run on mesh index ``mesh`` of a solver."""
    mach: float
    aoa_deg: float = 0.0
    mesh: int = 0
    cfl: float = 0.6
    tf: float = 4.0
    max_steps: int = 0
    gamma: float = 1.4
    rho_inf: float = 1.0
    p_inf: float = 1.0
    l_ref: float = 1.0
    clamp: bool = True
    dtype: type = np.float64
    eng_target_cd: float | None = None     # engineering criterion (euler/main.py:66-113)
    eng_target_cl: float | None = None
    eng_cd_tol: float = 0.001
    eng_cl_tol: float = 0.001
    eng_patience: int = 0                  # 0: the solver's stop-rule patience
    threshold: float | None = None         # this case's stop-rule threshold (None: the solver's)

    def to_c(self) -> F.Case:
        c = F.Case()
        c.mesh = int(self.mesh)
        c.mach = float(self.mach)
        c.aoa_deg = float(self.aoa_deg)
        c.cfl = float(clamp_cfl(self.mach, self.cfl) if self.clamp else self.cfl)
        c.tf = float(self.tf)
        c.max_steps = int(self.max_steps)
        c.inlet[:] = _freestream_values(float(self.mach), float(self.aoa_deg), float(self.gamma), float(self.rho_inf),
                                        float(self.p_inf), np.dtype(self.dtype).str)
        c.rho_inf = float(self.rho_inf)
        c.u_inf = float(self.mach * math.sqrt(self.gamma * self.p_inf / self.rho_inf))
        c.l_ref = float(self.l_ref)
        c.threshold = float(self.threshold) if self.threshold is not None else 0.0
        if self.eng_target_cd is not None and self.eng_target_cl is not None:
            c.eng_track = 1
            c.eng_patience = int(self.eng_patience)
            c.eng_target_cd = float(self.eng_target_cd)
            c.eng_target_cl = float(self.eng_target_cl)
            c.eng_cd_tol = float(self.eng_cd_tol)
            c.eng_cl_tol = float(self.eng_cl_tol)
        return c


# ------------------------------------------------------------------- mesh
class DeviceMesh:
    """A mesh prepared by the native library (renumbered, geometry in float64)."""

    def __init__(self, mesh: Mesh, renumber: bool = True, sponge: bool | None = None, sponge_width: float | None = None):
        L = F.lib()
        self.mesh = mesh
        self._keep = dict(points=F.f64(mesh.points), tris=F.i32(mesh.tris), neighbors=F.i32(mesh.neighbors),
                          faces=F.i32(mesh.faces), face_markers=F.i32(mesh.face_markers),
                          face_connectivity=F.i32(mesh.face_connectivity), walls=F.i32(mesh.wall_markers()))
        k = self._keep
        d = F.MeshDesc()
        d.n_points, d.n_cells, d.n_faces = len(k['points']), len(k['tris']), len(k['faces'])
        d.points = F.ptr(k['points'], C.c_double)
        d.tris = F.ptr(k['tris'], C.c_int32)
        d.neighbors = F.ptr(k['neighbors'], C.c_int32)
        d.faces = F.ptr(k['faces'], C.c_int32)
        d.face_markers = F.ptr(k['face_markers'], C.c_int32)
        d.face_connectivity = F.ptr(k['face_connectivity'], C.c_int32)
        d.wall_markers = F.ptr(k['walls'], C.c_int32)
        d.n_wall_markers = len(k['walls'])
        d.force_marker = mesh.force_marker()
        if sponge is None:
            sponge = mesh.metadata.get('case') != 'bump'
        d.sponge = int(bool(sponge))
        d.sponge_width = float(sponge_width or 0.0)
        sub = mesh.metadata.get('inlet_subsonic', [1.0, 1.0, 0.0, 1.0])
        for i in range(4):
            d.inlet_subsonic[i] = float(sub[i])
        d.renumber = int(bool(renumber))
        h = C.c_void_p()
        F.check(L.esr_mesh_create(C.byref(d), C.byref(h)))
        self.handle = h
        info = F.MeshInfo()
        F.check(L.esr_mesh_get_info(h, C.byref(info)))
        self.info = info

    @property
    def n_cells(self) -> int:
        return int(self.info.n_cells)

    def permutation(self) -> np.ndarray:
        perm = np.empty(self.n_cells, dtype=np.int32)
        F.check(F.lib().esr_mesh_get_permutation(self.handle, F.ptr(perm, C.c_int32)))
        return perm

    def patches(self) -> np.ndarray:
        """First new cell of every patch of the renumbering, plus n_cells."""
        n = C.c_int32()
        F.check(F.lib().esr_mesh_get_patches(self.handle, C.byref(n), None))
        start = np.empty(n.value + 1, dtype=np.int32)
        F.check(F.lib().esr_mesh_get_patches(self.handle, C.byref(n), F.ptr(start, C.c_int32)))
        return start

    def geometry(self, fidelity='fast', precision='f32'):
        """The per-cell records the kernels read (caller's cell order): a dict
        of normals (n,3,2), face lengths (n,3), area, blend3, lsq coefficients
        (n,3,2), face offsets (n,3,2) and, for reference fidelity in float32,
        the per-call least-squares data w (n,3), dx (n,3,2), A (n,2,2)."""
        n = self.n_cells
        geo = np.empty((n, 24), dtype=np.float64)
        lsq = np.empty((n, 13), dtype=np.float64)
        F.check(F.lib().esr_mesh_get_geometry(self.handle, F.FIDELITY[fidelity], F.PREC[precision],
                                              F.ptr(geo, C.c_double), F.ptr(lsq, C.c_double)))
        out = dict(normals=geo[:, 0:6].reshape(n, 3, 2), surface=geo[:, 6:9], area=geo[:, 9], blend3=geo[:, 10],
                   lsq_coef=geo[:, 12:18].reshape(n, 3, 2), face_offset=geo[:, 18:24].reshape(n, 3, 2))
        if fidelity == 'reference' and precision == 'f32':
            out.update(w=lsq[:, 0:3], dx=lsq[:, 3:9].reshape(n, 3, 2), A=lsq[:, 9:13].reshape(n, 2, 2))
        return out

    def close(self):
        if getattr(self, 'handle', None):
            F.lib().esr_mesh_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------- solver
class Solver:
    """All case slots of one or more meshes, advanced together on one GPU."""

    def __init__(self, meshes, slots, precision='f32', flux='hllc', reconstruction='muscl', time_scheme='SRK2',
                 dt_mode='global', stop_rule='reference', gamma=1.4, threshold=1e-6, check_every=25, patience=1,
                 device=0, use_graphs=True, block_size=0, fidelity='fast', stream_priority=0):
        L = F.lib()
        if isinstance(meshes, (DeviceMesh, Mesh)):
            meshes = [meshes]
        self.meshes = [m if isinstance(m, DeviceMesh) else DeviceMesh(m) for m in meshes]
        slots = [int(slots)] * len(self.meshes) if np.isscalar(slots) else [int(s) for s in slots]
        if len(slots) != len(self.meshes):
            raise ValueError("one slot count per mesh")
        p = F.Params()
        p.precision = F.PREC[str(precision).lower()]
        try:
            p.flux = F.FLUX[str(flux).lower()]
        except KeyError:
            raise ValueError(f"Unknown flux type '{flux}'.") from None
        try:
            p.reconstruction = F.RECON[str(reconstruction).lower()]
        except KeyError:
            raise ValueError(f"Unknown reconstruction scheme '{reconstruction}'. Expected 'constant' or 'muscl'.") from None
        p.time_scheme = F.TIME[str(time_scheme).upper()]
        p.dt_mode = F.DT_MODE[dt_mode]
        p.stop_rule = F.STOP_RULE[stop_rule]
        p.gamma = float(gamma)
        p.threshold = float(threshold)
        p.check_every = max(1, int(check_every))
        p.patience = max(1, int(patience))
        p.device = int(device)
        p.use_graphs = int(bool(use_graphs))
        p.block_size = F.BLOCK_PATCHES if block_size == "patches" else int(block_size)
        try:
            p.fidelity = F.FIDELITY[str(fidelity).lower()]
        except KeyError:
            raise ValueError(f"unknown fidelity '{fidelity}': expected 'fast' or 'reference'") from None
        p.stream_priority = int(stream_priority)
        self.params = p
        self.precision = 'f64' if p.precision == 1 else 'f32'
        self.dtype = np.float64 if p.precision == 1 else np.float32
        arr = (C.c_void_p * len(self.meshes))(*[m.handle for m in self.meshes])
        sl = np.asarray(slots, dtype=np.int32)
        h = C.c_void_p()
        F.check(L.esr_solver_create(arr, F.ptr(sl, C.c_int32), len(self.meshes), C.byref(p), C.byref(h)))
        self.handle = h
        n = C.c_int32()
        F.check(L.esr_solver_num_slots(h, C.byref(n)))
        self.n_slots = int(n.value)
        self.slots = slots
        self.slot_mesh = np.repeat(np.arange(len(slots)), slots)

    # ----------------------------------------------------------- state
    def _n_cells(self, slot):
        return self.meshes[int(self.slot_mesh[slot])].n_cells

    def set_case(self, slot: int, case: FlowCase, W_init=None):
        c = case.to_c()
        if W_init is not None:
            W = F.f64(W_init)
            if W.shape != (self._n_cells(slot), 4):
                raise ValueError(f"init field has shape {W.shape}, expected ({self._n_cells(slot)}, 4)")
            F.check(F.lib().esr_set_case(self.handle, slot, C.byref(c), F.ptr(W, C.c_double)))
        else:
            F.check(F.lib().esr_set_case(self.handle, slot, C.byref(c), None))

    def set_cases(self, slots, cases, W_inits=None):
        """set_case for many slots at once (one synchronisation). ``W_inits``:
        None or a list with an (n_cells, 4) field or None per slot. Fields that
        are all float32 go through the float32 entry point (half the bytes);
        pinned host arrays copy fastest."""
        n = len(slots)
        if len(cases) != n or (W_inits is not None and len(W_inits) != n):
            raise ValueError("set_cases: slots, cases and W_inits must have the same length")
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        carr = self._case_array(cases)
        given = [W for W in (W_inits or []) if W is not None]
        f32 = bool(given) and all(np.asarray(W).dtype == np.float32 for W in given)
        keep, arr = [], None
        if W_inits is not None:
            want = np.float32 if f32 else np.float64
            ncell = self._cells_of_slots(sl)
            addr = np.zeros(n, dtype=np.uintp)
            for i, W in enumerate(W_inits):
                if W is None:
                    continue
                W = np.ascontiguousarray(W, dtype=want)
                if W.shape != (ncell[i], 4):
                    raise ValueError(f"init field {i} has shape {W.shape}")
                keep.append(W)
                addr[i] = W.ctypes.data
            arr = addr.ctypes.data
        fn = F.lib().esr_set_cases_f32 if f32 else F.lib().esr_set_cases
        F.check(fn(self.handle, n, F.ptr(sl, C.c_int32), carr, arr))

    def _case_array(self, cases):
        """The C records of ``cases``, reused while every case's fields are
        unchanged (a serving loop re-submits the same cases)."""
        key = tuple(tuple(vars(c).values()) for c in cases)
        cached = getattr(self, "_carr_cache", None)
        if cached is not None and cached[0] == key:
            return cached[1]
        carr = (F.Case * len(cases))(*[c.to_c() for c in cases])
        self._carr_cache = (key, carr)
        return carr

    def _cells_of_slots(self, sl):
        ncell = getattr(self, "_slot_cells", None)
        if ncell is None:
            ncell = np.array([self.meshes[int(m)].n_cells for m in self.slot_mesh], dtype=np.int64)
            self._slot_cells = ncell
        return ncell[np.asarray(sl, dtype=np.int64)]

    def get_states(self, slots, out=None, dtype=np.float64):
        """get_state for many slots at once into ``out`` (C-contiguous
        (n_cells, 4) arrays of one dtype, float64 or float32; allocated with
        ``dtype`` when None); one synchronisation."""
        n = len(slots)
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        ncell = self._cells_of_slots(sl)
        if out is None:
            out = [np.empty((int(k), 4), dtype=dtype) for k in ncell]
        if len(out) != n:
            raise ValueError("get_states: one output array per slot")
        f32 = out[0].dtype == np.float32 if n else False
        want = np.float32 if f32 else np.float64
        addr = np.zeros(n, dtype=np.uintp)
        for i, o in enumerate(out):
            if o.shape != (ncell[i], 4) or o.dtype != want or not o.flags.c_contiguous:
                raise ValueError("get_states: outputs must be C-contiguous (n_cells, 4) arrays of one dtype")
            addr[i] = o.ctypes.data
        fn = F.lib().esr_get_states_f32 if f32 else F.lib().esr_get_states
        F.check(fn(self.handle, n, F.ptr(sl, C.c_int32), addr.ctypes.data))
        return out

    # ----------------------------------------------- overlapped transfers
    def stage_cases(self, slots, cases, fields):
        """Start uploading float32 fields (C-contiguous (n_cells, 4), pinned
        memory overlaps) for ``cases`` on ``slots`` and return; the arrays
        must stay unchanged until ``wait_transfers`` or the next stage_cases.
        ``apply_staged`` places them."""
        n = len(slots)
        if len(cases) != n or len(fields) != n:
            raise ValueError("stage_cases: slots, cases and fields must have the same length")
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        ncell = self._cells_of_slots(sl)
        addr = np.zeros(n, dtype=np.uintp)
        for i, W in enumerate(fields):
            if W.dtype != np.float32 or W.shape != (ncell[i], 4) or not W.flags.c_contiguous:
                raise ValueError("stage_cases: fields must be C-contiguous float32 (n_cells, 4) arrays")
            addr[i] = W.ctypes.data
        self._staged = (sl, fields)        # kept alive while the copy runs
        F.check(F.lib().esr_stage_cases_f32(self.handle, n, F.ptr(sl, C.c_int32), self._case_array(cases),
                                            addr.ctypes.data))

    def apply_staged(self):
        F.check(F.lib().esr_apply_staged(self.handle))

    def fetch_states(self, slots, out):
        """Gather the slots' fields after everything issued so far and start
        copying them into ``out`` (float32, C-contiguous (n_cells, 4)); returns
        at once. ``wait_transfers`` waits for the copy."""
        n = len(slots)
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        ncell = self._cells_of_slots(sl)
        if len(out) != n:
            raise ValueError("fetch_states: one output array per slot")
        addr = np.zeros(n, dtype=np.uintp)
        for i, o in enumerate(out):
            if o.dtype != np.float32 or o.shape != (ncell[i], 4) or not o.flags.c_contiguous:
                raise ValueError("fetch_states: outputs must be C-contiguous float32 (n_cells, 4) arrays")
            addr[i] = o.ctypes.data
        self._fetching = (sl, out)
        F.check(F.lib().esr_fetch_states_f32(self.handle, n, F.ptr(sl, C.c_int32), addr.ctypes.data))
        return out

    def wait_transfers(self):
        F.check(F.lib().esr_wait_transfers(self.handle))

    def set_state(self, slot: int, W):
        W = F.f64(W)
        if W.shape != (self._n_cells(slot), 4):
            raise ValueError("state shape mismatch")
        F.check(F.lib().esr_set_state(self.handle, slot, F.ptr(W, C.c_double)))

    def get_state(self, slot: int = 0) -> np.ndarray:
        out = np.empty((self._n_cells(slot), 4), dtype=np.float64)
        F.check(F.lib().esr_get_state(self.handle, slot, F.ptr(out, C.c_double)))
        return out

    def set_state_device(self, slot: int, ptr: int):
        F.check(F.lib().esr_set_state_device(self.handle, slot, C.c_void_p(ptr)))

    def get_state_device(self, slot: int, ptr: int):
        F.check(F.lib().esr_get_state_device(self.handle, slot, C.c_void_p(ptr)))

    def clear_slot(self, slot: int):
        F.check(F.lib().esr_clear_slot(self.handle, slot))

    # ------------------------------------------------------------ runs
    def dt(self) -> np.ndarray:
        out = np.empty(self.n_slots)
        F.check(F.lib().esr_compute_dt(self.handle, F.ptr(out, C.c_double)))
        return out

    def step(self, nsteps: int = 1):
        F.check(F.lib().esr_step(self.handle, int(nsteps)))

    def run(self) -> list[dict]:
        res = (F.Result * self.n_slots)()
        F.check(F.lib().esr_run(self.handle, res))
        return [r.as_dict() for r in res]

    def results(self) -> list[dict]:
        res = (F.Result * self.n_slots)()
        F.check(F.lib().esr_get_results(self.handle, res))
        return [r.as_dict() for r in res]

    def residual_probe(self) -> np.ndarray:
        out = np.empty(self.n_slots)
        F.check(F.lib().esr_residual_probe(self.handle, F.ptr(out, C.c_double)))
        return out

    def forces(self):
        cd = np.empty(self.n_slots)
        cl = np.empty(self.n_slots)
        F.check(F.lib().esr_forces(self.handle, F.ptr(cd, C.c_double), F.ptr(cl, C.c_double)))
        return cd, cl

    def gradients(self, slot: int = 0) -> np.ndarray:
        """(N, 4, 2) unlimited LSQ gradient of the primitives (bundle export)."""
        out = np.empty((self._n_cells(slot), 4, 2), dtype=np.float64)
        F.check(F.lib().esr_gradients(self.handle, slot, F.ptr(out, C.c_double)))
        return out

    def entropy(self) -> np.ndarray:
        out = np.empty(self.n_slots)
        F.check(F.lib().esr_entropy(self.handle, F.ptr(out, C.c_double)))
        return out

    def synchronize(self):
        F.check(F.lib().esr_synchronize(self.handle))

    def elapsed_ms(self) -> float:
        v = C.c_double()
        F.check(F.lib().esr_last_elapsed_ms(self.handle, C.byref(v)))
        return float(v.value)

    def kernel_launches(self) -> int:
        v = C.c_int64()
        F.check(F.lib().esr_kernel_launches(self.handle, C.byref(v)))
        return int(v.value)

    def tuning(self) -> dict:
        """Block size in use and, when autotuned, the step time per candidate."""
        t = F.Tuning()
        F.check(F.lib().esr_solver_tuning(self.handle, C.byref(t)))
        return t.as_dict()

    def set_shape(self, block_size: int, k2_patches: bool = False, k1_minb: int = 0, k2_minb: int = 0):
        """Run with this launch shape (one of ``tuning()['variants']``, say);
        a register budget of 0 is the kernel's default."""
        v = F.TuningVariant(block_size=int(block_size), k2_patches=int(bool(k2_patches)), k1_minb=int(k1_minb),
                            k2_minb=int(k2_minb), step_ms=0.0)
        F.check(F.lib().esr_solver_set_shape(self.handle, C.byref(v)))

    def profile_step(self, nsteps: int = 8) -> dict:
        """Average device ms per kernel kind over ``nsteps`` plain steps
        (CUDA events on the solver's stream around every launch)."""
        kt = F.KernelTimes()
        F.check(F.lib().esr_profile_step(self.handle, int(nsteps), C.byref(kt)))
        return kt.as_dict()

    def batch_solve(self, cases, init_fields=None, want_states=False):
        """Solve every case through the slots with retire/refill; returns
        (results, final states or None)."""
        n = len(cases)
        carr = (F.Case * n)(*[c.to_c() for c in cases])
        res = (F.Result * n)()
        init_arr, keep = self._init_array(cases, init_fields)
        fin_arr = None
        states = None
        if want_states:
            states = [np.empty((self.meshes[c.mesh].n_cells, 4)) for c in cases]
            fin_arr = (F._f64p * n)(*[F.ptr(s, C.c_double) for s in states])
        F.check(F.lib().esr_batch_solve(self.handle, carr, n, init_arr, fin_arr, res))
        return [r.as_dict() for r in res], states

    def _init_array(self, cases, init_fields):
        """Pointer array of the cases' float64 warm fields (None: freestream),
        each checked against its mesh's (n_cells, 4); the arrays to keep alive."""
        if init_fields is None:
            return None, []
        n = len(cases)
        if len(init_fields) != n:
            raise ValueError("one init field (or None) per case")
        arr, keep = (F._f64p * n)(), []
        for i, (c, f) in enumerate(zip(cases, init_fields)):
            if f is None:
                continue
            a = F.f64(f)
            if a.shape != (self.meshes[c.mesh].n_cells, 4):
                raise ValueError(f"init field {i} has shape {a.shape}, expected ({self.meshes[c.mesh].n_cells}, 4)")
            keep.append(a)
            arr[i] = F.ptr(a, C.c_double)
        return arr, keep

    def batch_submit(self, cases, init_fields=None, want_states=False):
        """Start the batch of ``batch_solve`` and return at once; the fields
        are copied before this returns. Until ``batch_results`` or
        ``batch_cancel`` the batch owns the slots."""
        n = len(cases)
        carr = (F.Case * n)(*[c.to_c() for c in cases])
        init_arr, keep = self._init_array(cases, init_fields)
        F.check(F.lib().esr_batch_submit(self.handle, carr, n, init_arr, int(bool(want_states))))
        self._pending = ([self.meshes[c.mesh].n_cells for c in cases], bool(want_states))

    def batch_poll(self) -> int:
        """Advance the submitted batch by a few chunks; returns the number of
        finished cases."""
        d = C.c_int32(0)
        try:
            F.check(F.lib().esr_batch_poll(self.handle, C.byref(d)))
        except Exception:
            self._pending = None   # a failing poll cancels the batch
            raise
        return int(d.value)

    def batch_results(self):
        """(results, final states or None) of the finished batch; releases it."""
        cells, want = self._pending
        n = len(cells)
        res = (F.Result * max(n, 1))()
        states = None
        fin_arr = None
        if want:
            states = [np.empty((nc, 4)) for nc in cells]
            fin_arr = (F._f64p * max(n, 1))(*[F.ptr(s, C.c_double) for s in states])
        F.check(F.lib().esr_batch_results(self.handle, fin_arr, res))
        self._pending = None
        return [r.as_dict() for r in res[:n]], states

    def batch_cancel(self):
        """Abandon the submitted batch: running cases stop, slots go inactive."""
        F.check(F.lib().esr_batch_cancel(self.handle))
        self._pending = None

    def close(self):
        if getattr(self, 'handle', None):
            F.lib().esr_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
