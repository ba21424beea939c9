"""Mesh model, mesher and file formats (CPU only)."""
import pickle
import sys
import types

import numpy as np
import pytest

from eulersr_b200.mesh import Mesh, load_reference_pickle, faces_neighbors_from_tris


@pytest.mark.parametrize("name", ["diamond_h0.2", "naca0012_h0.2", "diamond_h0.1"])
def test_golden_meshes_valid(name):
    from conftest import load_mesh
    m = load_mesh(name)
    assert m.validate()
    q = m.quality()
    assert q['min_angle_deg'] >= 29.9
    # markers: walls on the body, inlet on x=0, outlets elsewhere
    assert set(np.unique(m.face_markers)) == {0, 2, 3, 4}


def test_mesher_cell_counts_match_reference_scale():
    from eulersr_b200.meshing import build_mesh
    m = build_mesh('diamond', 0.1)
    assert 1200 <= m.n_cells <= 1700          # reference: ~1.4k cells at h=0.1
    assert m.quality()['min_angle_deg'] >= 29.9


def test_naca5_camber_and_naca4():
    from eulersr_b200.meshing import contours as C
    x = np.linspace(0, 1, 201)
    yc, dyc = C.naca5_camber(x, 0.3, 0.15)
    assert abs(yc.max() - 0.0184) < 2e-3        # NACA 23012: ~1.8% max camber near x=0.15
    assert abs(x[np.argmax(yc)] - 0.15) < 0.03
    t = C.naca_thickness(x, 0.12)
    assert abs(2 * t.max() - 0.12) < 1e-3 and abs(t[-1]) < 1e-12   # closed trailing edge
    yc4, _ = C.naca4_camber(x, 0.02, 0.4)
    assert abs(yc4.max() - 0.02) < 1e-4


def test_faces_neighbors_convention():
    tris = np.array([[0, 1, 2], [2, 1, 3]])
    faces, nb, fc, bnd = faces_neighbors_from_tris(tris)
    # edge 1 of tri 0 is (1,2) = edge 0 of tri 1 (2,1)
    assert nb[0, 1] == 1 and nb[1, 0] == 0
    assert fc[0, 1] == fc[1, 0]
    assert (nb < 0).sum() == 4


def test_graph_npz_roundtrip(tmp_path, diamond02):
    p = diamond02.save(tmp_path / "g.npz", W_snapshots={0.5: np.zeros((diamond02.n_cells, 4))},
                       inlet_state=[1, 2, 0, 3])
    d = np.load(p)
    for k in ("node_pos", "node_area", "edge_index", "edge_normals", "edge_lengths", "edge_vectors",
              "edge_face_index", "edge_bc_marker", "edge_kind", "bc_face_index", "bc_markers", "inlet_state",
              "t_0_5000"):
        assert k in d.files
    nint = int((diamond02.neighbors >= 0).sum())
    nb = int((diamond02.neighbors < 0).sum())
    assert d["edge_index"].shape == (2, nint + nb)
    m2 = Mesh.load(p)
    assert np.array_equal(m2.tris, diamond02.tris) and np.array_equal(m2.neighbors, diamond02.neighbors)
    assert np.allclose(m2.area, diamond02.area)
    assert m2.metadata['case'] == 'diamond'


def test_rcm_renumbering_preserves_geometry(diamond02):
    shuffled = diamond02.renumbered(np.random.default_rng(1).permutation(diamond02.n_cells))
    perm = shuffled.rcm_permutation()
    r = shuffled.renumbered(perm)
    assert r.validate()
    assert np.allclose(r.area, shuffled.area[perm])

    def bw(m):
        c, k = np.nonzero(m.neighbors >= 0)
        return np.abs(c - m.neighbors[c, k]).max()
    assert bw(r) < bw(shuffled) / 5


def test_wall_owner_first_listing_cell(diamond02):
    wf, wc, ws = diamond02.wall_owner_data()
    assert len(wf) > 0
    assert np.all(diamond02.face_connectivity[wc, ws] == wf)


def test_reference_pickle_reader(tmp_path, diamond02):
    """A pickle laid out like jnp.save of the reference Mesh (JAX array
    reconstructor + jax_fvm Mesh class) loads without JAX."""
    jarr = types.ModuleType("jax._src.array")

    def _reconstruct_array(fun, args, arr_state, aval_state):  # stand-in of JAX's own
        raise AssertionError("must not be called at load time")
    jarr._reconstruct_array = _reconstruct_array

    class FakeJaxArray:
        def __init__(self, a):
            self.a = np.asarray(a)

        def __reduce__(self):
            fun, args, state = self.a.__reduce__()
            return (_reconstruct_array, (fun, args, state, {'weak_type': False}))
    _reconstruct_array.__module__ = "jax._src.array"
    _reconstruct_array.__qualname__ = "_reconstruct_array"
    mod = types.ModuleType("jax_fvm.src.mesh")

    class Mesh_:  # the reference class name is Mesh
        pass
    Mesh_.__name__ = Mesh_.__qualname__ = "Mesh"
    Mesh_.__module__ = "jax_fvm.src.mesh"
    mod.Mesh = Mesh_
    saved = {k: sys.modules.get(k) for k in ("jax", "jax._src", "jax._src.array", "jax_fvm", "jax_fvm.src",
                                             "jax_fvm.src.mesh")}
    for k in ("jax", "jax._src", "jax_fvm", "jax_fvm.src"):
        sys.modules[k] = types.ModuleType(k)
    sys.modules["jax._src.array"] = jarr
    sys.modules["jax_fvm.src.mesh"] = mod
    try:
        obj = Mesh_()
        m = diamond02
        for key in ("points", "tris", "neighbors", "faces", "face_markers", "face_connectivity", "barycenter",
                    "area", "surface", "normals"):
            setattr(obj, key, FakeJaxArray(getattr(m, key)))
        obj.face_connectivity_opposite = FakeJaxArray(np.arange(m.n_faces))
        obj.metadata = {'case': 'diamond', 'h': 0.2}
        obj.chord = 1.0
        arr = np.empty((), dtype=object)
        arr[()] = obj
        path = tmp_path / "mesh.npy"
        with open(path, "wb") as f:
            np.lib.format.write_array(f, arr, allow_pickle=True)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    got = load_reference_pickle(path)
    assert np.array_equal(got.tris, diamond02.tris)
    assert np.array_equal(got.neighbors, diamond02.neighbors)
    assert got.metadata['obstacle_length'] == 1.0
    assert np.allclose(got.area, diamond02.area)


def test_generate_mesh_cli(tmp_path, capsys):
    """The euler/generate_mesh.py command line: --geom / -h / --out-dir give
    one <geom>_h<h>.npz per pair, placed as the reference places them."""
    import math
    from eulersr_b200.meshing import generate as G
    assert G.main(["--geom", "diamond_txy", "diamond_alpha10", "naca2412", "-h", "0.3",
                   "--out-dir", str(tmp_path), "--fig-dir", str(tmp_path / "figs")]) == 0
    out = capsys.readouterr().out
    assert out.count("Mesh saved : ") == 3
    txy = Mesh.load(tmp_path / "diamond_txy_h0.3.npz")
    assert txy.validate()
    assert txy.metadata["case"] == "diamond_txy"
    assert txy.metadata["center"] == {"cx": 2.0, "cy": 2.5}
    a10 = Mesh.load(tmp_path / "diamond_alpha10_h0.3.npz")
    assert math.isclose(a10.metadata["height"], math.tan(math.radians(10.0)))
    naca = Mesh.load(tmp_path / "naca2412_h0.3.npz")
    assert naca.metadata["case"] == "naca2412" and naca.n_cells > 0
    with pytest.raises(SystemExit):
        G.main(["--geom", "bump", "--out-dir", str(tmp_path)])
