"""ctypes binding of ``libeulersr.so`` (declarations in ``include/eulersr.h``).

Loading never falls back to anything: when the library is missing or fails to
load, :func:`lib` raises, so no solve can silently run elsewhere.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libeulersr.so"
HEADER = PKG.parent / "include" / "eulersr.h"

ESR_OK, ESR_ERR_ARG, ESR_ERR_CUDA, ESR_ERR_NONFINITE, ESR_ERR_TIMEOUT, ESR_ERR_OOM, ESR_ERR_STATE = range(7)
CASE_EMPTY, CASE_RUNNING, CASE_CONVERGED, CASE_MAXSTEP, CASE_NONFINITE = range(5)
STATUS_NAMES = {0: "empty", 1: "running", 2: "converged", 3: "maxstep", 4: "nonfinite"}
PREC = {"f32": 0, "float32": 0, "fp32": 0, "f64": 1, "float64": 1, "fp64": 1}
FLUX = {"hllc": 0, "hll": 0, "rusanov": 1}
RECON = {"muscl": 0, "second_order": 0, "2nd_order": 0, "constant": 1, "first_order": 1, "none": 1, "godunov": 1}
TIME = {"SRK2": 0, "SSP_RK2": 0, "EE": 1, "RK2": 2}
DT_MODE = {"global": 0, "local": 1}
STOP_RULE = {"reference": 0, "density_l2": 1, "engineering": 2}
FIDELITY = {"fast": 0, "reference": 1}

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class MeshDesc(C.Structure):
    _fields_ = [("n_points", C.c_int32), ("n_cells", C.c_int32), ("n_faces", C.c_int32),
                ("points", _f64p), ("tris", _i32p), ("neighbors", _i32p), ("faces", _i32p),
                ("face_markers", _i32p), ("face_connectivity", _i32p), ("wall_markers", _i32p),
                ("n_wall_markers", C.c_int32), ("force_marker", C.c_int32), ("sponge", C.c_int32),
                ("sponge_width", C.c_double), ("inlet_subsonic", C.c_double * 4), ("renumber", C.c_int32)]


class MeshInfo(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_wall_faces", C.c_int32),
                ("n_boundary_slots", C.c_int32), ("y_min", C.c_double), ("y_max", C.c_double),
                ("device_bytes_f32", C.c_int64), ("device_bytes_f64", C.c_int64)]


class Params(C.Structure):
    _fields_ = [("precision", C.c_int32), ("flux", C.c_int32), ("reconstruction", C.c_int32),
                ("time_scheme", C.c_int32), ("dt_mode", C.c_int32), ("stop_rule", C.c_int32),
                ("gamma", C.c_double), ("threshold", C.c_double), ("check_every", C.c_int32),
                ("patience", C.c_int32), ("device", C.c_int32), ("use_graphs", C.c_int32),
                ("block_size", C.c_int32), ("fidelity", C.c_int32), ("stream_priority", C.c_int32)]


class Case(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("reserved", C.c_int32), ("mach", C.c_double), ("aoa_deg", C.c_double),
                ("cfl", C.c_double), ("tf", C.c_double), ("max_steps", C.c_int64), ("inlet", C.c_double * 4),
                ("rho_inf", C.c_double), ("u_inf", C.c_double), ("l_ref", C.c_double),
                ("eng_track", C.c_int32), ("eng_patience", C.c_int32), ("eng_target_cd", C.c_double),
                ("eng_target_cl", C.c_double), ("eng_cd_tol", C.c_double), ("eng_cl_tol", C.c_double),
                ("threshold", C.c_double)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("converged", C.c_int32), ("stopping_step", C.c_int32),
                ("steps", C.c_int32), ("n_max", C.c_int32), ("case_index", C.c_int32), ("dt", C.c_double),
                ("last_rel", C.c_double), ("cd", C.c_double), ("cl", C.c_double), ("solve_time_s", C.c_double),
                ("eng_converged", C.c_int32), ("eng_stopping_step", C.c_int32), ("final_residual", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class KernelTimes(C.Structure):
    _fields_ = [("recon_ms", C.c_double), ("flux_ms", C.c_double), ("other_ms", C.c_double),
                ("recon_launches", C.c_int32), ("flux_launches", C.c_int32), ("other_launches", C.c_int32),
                ("reserved", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


BLOCK_PATCHES = -1


TUNING_MAX_VARIANTS = 12


class TuningVariant(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("k2_patches", C.c_int32), ("k1_minb", C.c_int32),
                ("k2_minb", C.c_int32), ("step_ms", C.c_double)]

    def as_dict(self):
        return {"block_size": int(self.block_size), "k2_patches": bool(self.k2_patches),
                "k1_minb": int(self.k1_minb), "k2_minb": int(self.k2_minb), "step_ms": float(self.step_ms)}


class Tuning(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("n_candidates", C.c_int32), ("candidates", C.c_int32 * 4),
                ("k2_patches", C.c_int32), ("cached", C.c_int32), ("step_ms", C.c_double * 4),
                ("k1_minb", C.c_int32), ("k2_minb", C.c_int32), ("n_variants", C.c_int32),
                ("reserved", C.c_int32), ("variants", TuningVariant * TUNING_MAX_VARIANTS)]

    def as_dict(self):
        n = int(self.n_candidates)
        name = lambda c: "patches" if c == BLOCK_PATCHES else int(c)
        return {"block_size": int(self.block_size), "k2_patches": bool(self.k2_patches),
                "k1_minb": int(self.k1_minb), "k2_minb": int(self.k2_minb), "cached": bool(self.cached),
                "step_ms": {name(self.candidates[i]): float(self.step_ms[i]) for i in range(n)},
                "variants": [self.variants[i].as_dict() for i in range(int(self.n_variants))]}


class EsrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"eulersr error {code}: {msg}")
        self.code = code


_LIB = None

_GEMM_ARGS = [C.c_int32] * 5 + [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]

_SIGS = {
    "esr_api_version": (C.c_int32, []),
    "esr_last_error": (C.c_char_p, []),
    "esr_mesh_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(C.c_void_p)]),
    "esr_mesh_destroy": (C.c_int, [C.c_void_p]),
    "esr_mesh_get_info": (C.c_int, [C.c_void_p, C.POINTER(MeshInfo)]),
    "esr_mesh_get_permutation": (C.c_int, [C.c_void_p, _i32p]),
    "esr_mesh_get_geometry": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "esr_mesh_get_patches": (C.c_int, [C.c_void_p, _i32p, C.c_void_p]),
    "esr_stage_cases_f32": (C.c_int, [C.c_void_p, C.c_int32, _i32p, C.c_void_p, C.c_void_p]),
    "esr_apply_staged": (C.c_int, [C.c_void_p]),
    "esr_fetch_states_f32": (C.c_int, [C.c_void_p, C.c_int32, _i32p, C.c_void_p]),
    "esr_wait_transfers": (C.c_int, [C.c_void_p]),
    "esr_solver_create": (C.c_int, [C.POINTER(C.c_void_p), _i32p, C.c_int32, C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "esr_solver_destroy": (C.c_int, [C.c_void_p]),
    "esr_solver_num_slots": (C.c_int, [C.c_void_p, _i32p]),
    "esr_set_case": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Case), _f64p]),
    "esr_clear_slot": (C.c_int, [C.c_void_p, C.c_int32]),
    "esr_set_state": (C.c_int, [C.c_void_p, C.c_int32, _f64p]),
    "esr_get_state": (C.c_int, [C.c_void_p, C.c_int32, _f64p]),
    "esr_set_state_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "esr_get_state_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "esr_compute_dt": (C.c_int, [C.c_void_p, _f64p]),
    "esr_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "esr_run": (C.c_int, [C.c_void_p, C.POINTER(Result)]),
    "esr_get_results": (C.c_int, [C.c_void_p, C.POINTER(Result)]),
    "esr_residual_probe": (C.c_int, [C.c_void_p, _f64p]),
    "esr_forces": (C.c_int, [C.c_void_p, _f64p, _f64p]),
    "esr_entropy": (C.c_int, [C.c_void_p, _f64p]),
    "esr_gradients": (C.c_int, [C.c_void_p, C.c_int32, _f64p]),
    "esr_synchronize": (C.c_int, [C.c_void_p]),
    "esr_last_elapsed_ms": (C.c_int, [C.c_void_p, _f64p]),
    "esr_kernel_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "esr_profile_step": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "esr_solver_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "esr_solver_set_shape": (C.c_int, [C.c_void_p, C.POINTER(TuningVariant)]),
    "esr_set_cases": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(Case), C.c_void_p]),
    "esr_get_states": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "esr_set_cases_f32": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(Case), C.c_void_p]),
    "esr_get_states_f32": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "esr_batch_solve": (C.c_int, [C.c_void_p, C.POINTER(Case), C.c_int32, C.POINTER(_f64p), C.POINTER(_f64p),
                                  C.POINTER(Result)]),
    "esr_batch_submit": (C.c_int, [C.c_void_p, C.POINTER(Case), C.c_int32, C.POINTER(_f64p), C.c_int32]),
    "esr_batch_poll": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "esr_batch_results": (C.c_int, [C.c_void_p, C.POINTER(_f64p), C.POINTER(Result)]),
    "esr_batch_cancel": (C.c_int, [C.c_void_p]),
    "esr_gemm_bf16": (C.c_int, _GEMM_ARGS),
    "esr_gemm_bf16_mma_sync": (C.c_int, _GEMM_ARGS),
    "esr_gemm_tc_status": (C.c_int, [C.POINTER(C.c_int32)]),
    "esr_mlp_head_fwd": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    "esr_mlp_head_bwd": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "esr_mlp_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_float,
                                   C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "esr_mlp_decode": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float,
                                 C.c_void_p, C.c_void_p]),
    "esr_mlp_loss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p]),
    "esr_reduce_splits": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]),
    "esr_colsum_bf16": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "esr_adamw": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float,
                            C.c_float, C.c_float, C.c_float, C.c_int32, C.c_void_p, C.c_void_p]),
    "esr_rel_change_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]),
    "esr_idw_apply": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                C.c_void_p, C.c_void_p]),
    "esr_idw_status": (C.c_int, [C.POINTER(C.c_int32)]),
}


def header_functions() -> list[str]:
    """Names of every function ``include/eulersr.h`` declares."""
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(esr_[a-z0-9_]+)\s*\(", txt)))


def lib():
    """Load the library (building it first when the sources are newer)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        try:
            from . import _build
            _build.build()
        except Exception as e:  # pragma: no cover - depends on the toolchain
            raise RuntimeError(f"libeulersr.so is missing and could not be built: {e}") from e
    L = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def check(rc: int):
    if rc != ESR_OK:
        msg = lib().esr_last_error()
        raise EsrError(rc, msg.decode() if msg else "")


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))
