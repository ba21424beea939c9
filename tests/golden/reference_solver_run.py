"""Run EulerSR's own solver source on a golden mesh with NumPy in place of
jax.numpy (JAX is not installed), for the fixture ``reference_solver.npz``.

The functions are compiled from the reference's source text (no module of the
reference is imported, so none of its plotting or meshing dependencies is
needed): the mesh geometry methods of ``euler/jax_fvm/src/mesh.py:223-264``,
the helpers of ``euler/jax_fvm/src/helper.py`` (conversions, dt, LSQ
gradient, boundary states, sponge), the solver of
``euler/jax_fvm/src/euler_solver.py`` (limiter, MUSCL, reconstruction, HLLC,
getFlux, residual, SRK2) and ``initialize`` of ``euler/main.py:28-41``.
What stands in for JAX:

* ``jnp``: NumPy, with array results given an ``.at[...].set()`` that
  returns an updated copy, and, in single precision, new float arrays made
  float32 as JAX does without ``JAX_ENABLE_X64``;
* ``jax.jit``: the identity; ``jax.lax.cond``: a Python branch;
  ``jax.vmap``: a loop over the leading axis.

Used by ``make_reference_fixtures.py``.
"""
from __future__ import annotations

import ast
import functools
import types
from pathlib import Path

import numpy as np


class _JArr(np.ndarray):
    @property
    def at(self):
        return _At(self)


class _At:
    def __init__(self, a):
        self.a = a

    def __getitem__(self, idx):
        return _AtIdx(self.a, idx)


class _AtIdx:
    def __init__(self, a, idx):
        self.a, self.idx = a, idx

    def set(self, v):
        c = np.array(self.a, copy=True).view(_JArr)
        c[self.idx] = v
        return c


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, _JArr):
        return x.view(_JArr)
    return x


class _NumpyAsJnp:
    def __init__(self, mod, float32):
        self._mod, self._f32 = mod, float32

    def __getattr__(self, name):
        if name == "linalg":
            return _NumpyAsJnp(np.linalg, self._f32)
        attr = getattr(self._mod, name)
        if isinstance(attr, type) or not callable(attr):
            return attr
        make = name in ("asarray", "array", "zeros", "ones", "full", "arange", "linspace")

        def call(*a, **k):
            out = attr(*a, **k)
            if make and self._f32 and "dtype" not in k and isinstance(out, np.ndarray) and out.dtype == np.float64:
                out = out.astype(np.float32)
            return _wrap(out)
        return call


def _vmap(f):
    def g(*args):
        outs = [f(*[a[i] for a in args]) for i in range(args[0].shape[0])]
        if outs and isinstance(outs[0], tuple):
            return tuple(_wrap(np.stack([o[j] for o in outs])) for j in range(len(outs[0])))
        return _wrap(np.stack(outs))
    return g


class _Jitted:
    """jax.jit: calls the function; .lower(x).compile() gives it back."""

    def __init__(self, f, **kw):
        self.f = f

    def __call__(self, *a, **k):
        return self.f(*a, **k)

    def lower(self, *a, **k):
        return types.SimpleNamespace(compile=lambda: self.f)


def _jit(f=None, **kw):
    return _Jitted(f, **kw) if f is not None else (lambda g: _Jitted(g, **kw))


def _scan(body, carry, xs, length=None):
    """jax.lax.scan as a loop (no per-step outputs are used here)."""
    for _ in range(length):
        carry, _ = body(carry, None)
    return carry, None


def _jax(jnp):
    lax = types.SimpleNamespace(cond=lambda p, t, f, operand=None: t(operand) if bool(p) else f(operand),
                                scan=_scan)
    return types.SimpleNamespace(jit=_jit, lax=lax, vmap=_vmap, numpy=jnp, block_until_ready=lambda x: x)


def _defs(path: Path, names, cls=None):
    tree = ast.parse(path.read_text())
    body = tree.body
    if cls is not None:
        body = next(n for n in body if isinstance(n, ast.ClassDef) and n.name == cls).body
    found = [n for n in body if isinstance(n, ast.FunctionDef) and n.name in names]
    assert {n.name for n in found} == set(names), set(names) - {n.name for n in found}
    return found


def _compile(nodes, ns, filename):
    exec(compile(ast.Module(body=nodes, type_ignores=[]), filename, "exec"), ns)
    return ns


def _setup(ref_root, mesh, dtype, aoa_cases, known_cases=(), format_snapshot_name=None):
    src = Path(ref_root) / "euler"
    f32 = dtype == np.float32
    jnp = _NumpyAsJnp(np, f32)
    jax = _jax(jnp)
    base = {"jnp": jnp, "jax": jax, "np": np, "partial": functools.partial}
    geo = _compile(_defs(src / "jax_fvm" / "src" / "mesh.py",
                         ["getCenterTriangles", "getNormals", "getArea", "getSurface", "get_face_connectivity"],
                         cls="Mesh"), dict(base), "mesh.py")
    M = types.SimpleNamespace()
    M.points = _wrap(np.asarray(mesh.points, dtype=dtype))
    M.tris = np.asarray(mesh.tris, dtype=np.int32)
    M.faces = np.asarray(mesh.faces, dtype=np.int32)
    for meth in ("getCenterTriangles", "getNormals", "getArea", "getSurface", "get_face_connectivity"):
        geo[meth](M)
    M.neighbors = np.asarray(mesh.neighbors, dtype=np.int32)
    M.face_markers = np.asarray(mesh.face_markers, dtype=np.int32)
    M.face_connectivity_opposite = np.arange(M.faces.shape[0])
    M.metadata = dict(mesh.metadata)
    M.inlet_subsonic = jnp.array([1.0, 1., 0.0, 1.0])
    helper_names = ["get_dt", "getConserved", "getPrimitive", "getgradientLSQ", "BC_outflow", "BC_inflow",
                    "BC_subsonic_inlet", "BC_slipwall", "_mesh_metadata", "BC_state", "get_sponge_source",
                    "get_drag_coefficient", "get_lift_coefficient", "get_specific_entropy", "get_total_entropy",
                    "get_entropy_creation"]
    hns = _compile(_defs(src / "jax_fvm" / "src" / "helper.py", helper_names), dict(base), "helper.py")
    helper = types.SimpleNamespace(**{k: hns[k] for k in helper_names})
    solver_names = ["venkatakrishnan", "getlimiting", "MUSCL", "get_reconstruction_mode", "get_flux_type",
                    "build_reconstruction", "build_flux", "apply_face_surfaces", "Rusanov", "HLLC", "getFlux",
                    "residual", "time_step_Euler", "time_step_RK2_SSP", "time_step_RK2", "time_step_RK4"]
    sns = _compile(_defs(src / "jax_fvm" / "src" / "euler_solver.py", solver_names),
                   dict(base, helper=helper), "euler_solver.py")
    euler = types.SimpleNamespace(**{k: sns[k] for k in solver_names})
    import time as _time
    mns = _compile(_defs(src / "main.py", ["initialize", "run"]),
                   dict(base, helper=helper, euler=euler, time=_time, _AOA_CASES_LC=tuple(aoa_cases),
                        _KNOWN_CASES_LC=tuple(known_cases), format_snapshot_name=format_snapshot_name),
                   "main.py")
    return M, helper, sns, mns


def run_main(ref_root, mesh, cfg, dtype, aoa_cases, known_cases, format_snapshot_name):
    """euler/main.py:43-270 itself (stop rule, engineering criterion, final
    probe) with all exports off; returns (W, final carry of the loop)."""
    M, helper, sns, mns = _setup(ref_root, mesh, dtype, aoa_cases, known_cases, format_snapshot_name)
    W, inlet = mns["initialize"](M, cfg)
    captured = {}
    scan0 = mns["jax"].lax.scan

    def scan(body, carry, xs, length=None):
        out = scan0(body, carry, xs, length=length)
        captured["carry"] = out[0]
        return out
    mns["jax"].lax.scan = scan
    cfg = dict(cfg, export=dict(results=False, figures=False, graph=False, summary=False, bundle=False, n_snaps=1),
               verbose=False)
    W = mns["run"](W, M, inlet, cfg, {})
    return np.asarray(W), captured["carry"]


def run(ref_root, mesh, mach, aoa, steps, dtype, aoa_cases, flux="HLLC", reconstruction="MUSCL",
        scheme="SRK2", diagnostics=False):
    """(W after `steps` steps of `scheme`, dt) of the reference code on `mesh`
    (an object with points, tris, faces, face_markers, neighbors, metadata);
    with diagnostics, also the reference's CD, CL (helper.py:366-415) and the
    entropy created since the start (helper.py:312-320) of the final state."""
    M, helper, sns, mns = _setup(ref_root, mesh, dtype, aoa_cases)
    cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=mach, aoa=aoa, case=mesh.metadata["case"], CFL=0.6)
    if 0.6 < cfg["Mach"] < 1.1 and cfg["CFL"] > 0.45:     # euler/main.py:117-120
        cfg["CFL"] = 0.45
    W0, inlet = mns["initialize"](M, cfg)
    dt = helper.get_dt(W0, M, CFL=cfg["CFL"], gamma=cfg["gamma"], M=1.0)
    fn = {"EE": sns["time_step_Euler"], "RK2": sns["time_step_RK2"], "SRK2": sns["time_step_RK2_SSP"]}[scheme]
    kw = dict(gamma=cfg["gamma"], M=1.0, reconstruction=reconstruction, flux=flux, value=inlet, entropy=False)
    W = W0
    for _ in range(steps):
        W = fn(W, M, dt, **kw)
    if not diagnostics:
        return np.asarray(W), float(dt)
    u_inf = mach * float(np.sqrt(1.4 * 1.0 / 1.0))
    L = mesh.metadata["obstacle_length"]
    cd = helper.get_drag_coefficient(W=W, mesh=M, rho_inf=1.0, U_inf=u_inf, L_ref=L)
    cl = helper.get_lift_coefficient(W=W, mesh=M, rho_inf=1.0, U_inf=u_inf, L_ref=L)
    ds = helper.get_entropy_creation(W0, W, M, gamma=1.4)
    return np.asarray(W), float(dt), float(cd), float(cl), float(ds)
