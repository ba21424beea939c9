"""Parity on the HR meshes (h = 0.025), float32 rounded as the reference rounds it.

Config 2: the diamond at h = 0.025 (the package's mesher, 19,384 cells),
M 2.0, alpha 0, CFL 0.6; and the NACA0012 h = 0.025 mesh of the batched
workload (25,049 cells), transonic M 0.8, alpha 1.25 (CFL 0.45).

* float32 with ``fidelity='reference'`` (geometry formed in float32 in the
  reference's operation order, the least-squares gradient solved per call,
  IEEE division, no fused multiply-add): within 1e-5 per field of the
  oracle's float32 after 100 SRK2 steps. The oracle is the reference's
  float32 arithmetic (it equals the reference's source run with NumPy bit
  for bit, tests/test_reference_fixtures.py).
* float64 within 1e-12 of the oracle's float64 after 100 steps (diamond).
* directly against the reference's own source on the HR diamond
  (tests/golden/reference_solver_hr.npz, 20 steps, float32 and float64).
* converged force coefficients: the float32 run (reference fidelity) stopped
  by the reference rule (threshold 1e-5, checked every 25 steps) against the
  float64 build of the same kernels advanced the same number of steps:
  CD within 1e-4 relative, CL within 1e-5 absolute (CL is ~0 at alpha 0).

Why the float32 bar needs the reference's rounding: on the HR diamond the
reference's own float32 field moves by ~1.5e-5 after 100 steps when its state
gets 0.5-ulp random noise per step (the limiter's switches amplify rounding),
so a float32 path that rounds differently cannot stay within 1e-5 of it.
The fast float32 path (geometry from float64, approximate division) is
reported beside it, not held to 1e-5.
"""
import numpy as np
import pytest

from conftest import GOLDEN, oracle_mesh, rel_err

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
TOL64 = 1e-12
CASES = {"diamond": (2.0, 0.0), "naca0012": (0.8, 1.25)}


@pytest.fixture(scope="module")
def hr_meshes():
    from eulersr_b200.meshing.generate import cached_mesh
    return {g: cached_mesh(g, 0.025) for g in CASES}


_oracle_cache = {}


def _oracle(mesh, geom, dtype, steps):
    key = (geom, np.dtype(dtype).name, steps)
    if key not in _oracle_cache:
        from oracle import euler_oracle as O
        mach, aoa = CASES[geom]
        om = oracle_mesh(mesh, dtype)
        W, inlet = O.initialize(mesh.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=mach, aoa=aoa,
                                                   case=mesh.metadata["case"]), dtype)
        dt = O.get_dt(W, om, CFL=0.45 if 0.6 < mach < 1.1 else 0.6)
        for _ in range(steps):
            W = O.time_step_srk2(W, om, dt, inlet)
        _oracle_cache[key] = (W, dt)
    return _oracle_cache[key]


def _gpu(mesh, geom, prec, steps, fidelity):
    from eulersr_b200.solver import Solver, FlowCase
    mach, aoa = CASES[geom]
    dtype = np.float64 if prec == "f64" else np.float32
    s = Solver(mesh, 1, precision=prec, fidelity=fidelity)
    s.set_case(0, FlowCase(mach=mach, aoa_deg=aoa, cfl=0.6, tf=1e9, dtype=dtype))
    dt = s.dt()[0]
    s.step(steps)
    W = s.get_state(0)
    s.close()
    return W, dt


@pytest.mark.parametrize("geom", ["diamond", "naca0012"])
def test_hr_f32_reference_fidelity_100_steps(hr_meshes, geom):
    mesh = hr_meshes[geom]
    Wo, dto = _oracle(mesh, geom, np.float32, 100)
    Wg, dtg = _gpu(mesh, geom, "f32", 100, "reference")
    Wf, _ = _gpu(mesh, geom, "f32", 100, "fast")
    e_ref, e_fast = rel_err(Wg, Wo), rel_err(Wf, Wo)
    print(f"{geom} h=0.025 ({mesh.n_cells} cells), 100 SRK2 steps vs the oracle's float32: "
          f"reference fidelity {e_ref:.3e} (bitwise equal cells {np.mean(np.all(Wg == Wo, axis=1)):.4f}), "
          f"fast {e_fast:.3e}")
    assert float(dtg) == float(dto)
    assert e_ref <= TOL32, e_ref


def test_hr_diamond_f64_100_steps(hr_meshes):
    mesh = hr_meshes["diamond"]
    Wo, dto = _oracle(mesh, "diamond", np.float64, 100)
    Wg, dtg = _gpu(mesh, "diamond", "f64", 100, "fast")
    assert abs(dtg - dto) <= 1e-14 * dto
    assert rel_err(Wg, Wo) <= TOL64
    Wr, _ = _gpu(mesh, "diamond", "f64", 100, "reference")
    assert rel_err(Wr, Wo) <= TOL64


def test_hr_diamond_against_reference_source(hr_meshes):
    """The reference's own solver source, run with NumPy on this very mesh."""
    from golden.make_reference_fixtures import mesh_digest
    mesh = hr_meshes["diamond"]
    ref = np.load(GOLDEN / "reference_solver_hr.npz")
    assert str(ref["mesh_sha256"]) == mesh_digest(mesh)
    W32, dt32 = _gpu(mesh, "diamond", "f32", 20, "reference")
    assert float(dt32) == float(ref["f32_dt"])
    e32 = rel_err(W32, ref["f32_W20"])
    W64, dt64 = _gpu(mesh, "diamond", "f64", 20, "fast")
    e64 = rel_err(W64, ref["f64_W20"])
    print(f"HR diamond vs the reference's source after 20 steps: float32 {e32:.3e}, float64 {e64:.3e}")
    assert e32 <= TOL32
    assert abs(dt64 - float(ref["f64_dt"])) <= 1e-14 * float(ref["f64_dt"])
    assert e64 <= TOL64


def test_hr_diamond_converged_forces_f32_vs_f64(hr_meshes):
    from eulersr_b200.solver import Solver, FlowCase
    mesh = hr_meshes["diamond"]
    mach, aoa = CASES["diamond"]
    s = Solver(mesh, 1, precision="f32", fidelity="reference", threshold=1e-5, check_every=25, patience=1)
    s.set_case(0, FlowCase(mach=mach, aoa_deg=aoa, cfl=0.6, tf=1e9, max_steps=40000, dtype=np.float32))
    r = s.run()[0]
    s.close()
    assert r["converged"], r
    n = int(r["steps"])
    d = Solver(mesh, 1, precision="f64")
    d.set_case(0, FlowCase(mach=mach, aoa_deg=aoa, cfl=0.6, tf=1e9, dtype=np.float64))
    d.step(n)
    cd, cl = d.forces()
    d.close()
    print(f"HR diamond converged in {n} steps: float32 CD {r['cd']:.7f} CL {r['cl']:.2e}, "
          f"float64 CD {cd[0]:.7f} CL {cl[0]:.2e}")
    assert abs(r["cd"] - cd[0]) <= 1e-4 * abs(cd[0])
    # CL is zero by symmetry at alpha 0 (the mesh leaves ~3e-4): relative
    # error means nothing there, so it is held to 1e-5 absolute
    assert abs(r["cl"] - cl[0]) <= 1e-5
