"""The reference-fidelity geometry (no GPU needed): the records the float32
kernels read with ``fidelity='reference'`` equal, bit for bit, the geometry
the oracle forms in float32 as the reference forms it on every call
(mesh.py:223-240 normals, face lengths and areas; euler_solver.py:49,74,79
face offsets; helper.py:136-150 least-squares offsets, weights and matrix;
the oracle itself equals the reference's source run with NumPy bit for bit).
The sponge blend^3 is held to 1 ulp: NumPy's float32 power may use its own
SIMD routine where the library calls powf. The fast fidelity's float64
geometry is checked against the oracle's float64 to a few ulp.
"""
import numpy as np
import pytest

from conftest import oracle_mesh


def _oracle_parts(mesh, dtype):
    from oracle import euler_oracle as O
    om = oracle_mesh(mesh, dtype)
    mk = O._face_marker_slots(om)
    mid = O.face_midpoints(om)
    offs = mid - om.barycenter[..., None, :]
    dx = om.barycenter[om.neighbors] - om.barycenter[..., None, :]
    dx = np.where((mk > 0)[..., None], dtype(2) * offs, dx)
    w = 1 / np.linalg.norm(dx, axis=-1) ** 2
    A = np.einsum('ijk,ijl->ikl', w[..., None] * dx, dx)
    y = om.barycenter[:, 1]
    y_min, y_max = np.min(om.points[:, 1]), np.max(om.points[:, 1])
    width = dtype(0.2) * (y_max - y_min)
    blend = np.clip((width - np.minimum(y - y_min, y_max - y)) / width, dtype(0), dtype(1)) ** 3
    return dict(normals=om.normals, surface=om.surface[om.face_connectivity], area=om.area, face_offset=offs,
                w=w, dx=dx, A=A, blend3=blend)


@pytest.mark.parametrize("name", ["diamond_h0.2", "naca0012_h0.2", "diamond_h0.1"])
def test_reference_fidelity_geometry_is_the_oracles_float32(name):
    from conftest import load_mesh
    from eulersr_b200.solver import DeviceMesh
    mesh = load_mesh(name)
    dm = DeviceMesh(mesh)
    g = dm.geometry("reference", "f32")
    o = _oracle_parts(mesh, np.float32)
    for key in ("normals", "surface", "area", "face_offset", "w", "dx", "A"):
        got = g[key].astype(np.float32)
        assert np.array_equal(got, o[key]), (key, np.max(np.abs(got - o[key])))
    b = g["blend3"].astype(np.float32)
    ulp = np.spacing(np.maximum(np.abs(o["blend3"]), np.float32(1e-30)))
    assert np.all(np.abs(b - o["blend3"]) <= ulp)
    dm.close()


def test_fast_fidelity_geometry_is_float64():
    from conftest import load_mesh
    from eulersr_b200.solver import DeviceMesh
    mesh = load_mesh("diamond_h0.2")
    dm = DeviceMesh(mesh)
    g = dm.geometry("fast", "f64")
    o = _oracle_parts(mesh, np.float64)
    for key in ("normals", "surface", "area", "face_offset"):
        assert np.allclose(g[key], o[key], rtol=4e-16 * 8, atol=1e-16), key
    r = dm.geometry("reference", "f64")
    for key in ("normals", "surface", "area", "face_offset"):
        assert np.array_equal(r[key], o[key]), key
    dm.close()
