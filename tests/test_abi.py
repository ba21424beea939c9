"""The C ABI library: loads, exports every declared symbol, prepares meshes on
the host and rejects bad input with the reference's error classes (CPU only;
no compute call needs a GPU here)."""
import ctypes as C

import numpy as np
import pytest


def test_library_exports_every_header_symbol():
    from eulersr_b200 import _ffi as F
    L = F.lib()
    names = F.header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.esr_api_version() == 1


def test_mesh_prepare_on_host(diamond02):
    from eulersr_b200.solver import DeviceMesh
    dm = DeviceMesh(diamond02)
    assert dm.n_cells == diamond02.n_cells
    perm = dm.permutation()
    assert np.array_equal(np.sort(perm), np.arange(diamond02.n_cells))
    wf, _, _ = diamond02.wall_owner_data()
    assert dm.info.n_wall_faces == len(wf)
    assert dm.info.n_boundary_slots == int((diamond02.neighbors < 0).sum())
    assert dm.info.y_min == pytest.approx(0.0) and dm.info.y_max == pytest.approx(4.0)


def test_mesh_rejects_periodic_marker(diamond02):
    from eulersr_b200 import _ffi as F
    from eulersr_b200.mesh import Mesh
    from eulersr_b200.solver import DeviceMesh
    fm = diamond02.face_markers.copy()
    fm[fm == 4] = 1
    bad = Mesh.from_arrays(diamond02.points, diamond02.tris, diamond02.neighbors, diamond02.faces, fm,
                           diamond02.face_connectivity, dict(diamond02.metadata))
    with pytest.raises(F.EsrError) as e:
        DeviceMesh(bad)
    assert e.value.code == F.ESR_ERR_ARG and "periodic" in str(e.value)


def test_mesh_rejects_out_of_range(diamond02):
    from eulersr_b200 import _ffi as F
    from eulersr_b200.mesh import Mesh
    from eulersr_b200.solver import DeviceMesh
    nb = diamond02.neighbors.copy()
    nb[0, 0] = diamond02.n_cells + 5
    bad = Mesh.__new__(Mesh)
    bad.__dict__.update(diamond02.__dict__)
    bad.neighbors = nb
    with pytest.raises(F.EsrError) as e:
        DeviceMesh(bad)
    assert e.value.code == F.ESR_ERR_ARG


def test_solver_argument_errors_before_cuda(diamond02):
    """Unknown flux / reconstruction names fail like the reference's
    ValueError (euler_solver.py:122,139) without touching the device."""
    from eulersr_b200.solver import Solver
    with pytest.raises(ValueError, match="Unknown flux type"):
        Solver(diamond02, 1, flux="roe")
    with pytest.raises(ValueError, match="Unknown reconstruction scheme"):
        Solver(diamond02, 1, reconstruction="weno")


def test_renumbering_contract(diamond02):
    """The library's renumbering is a permutation that keeps neighbours close
    (compact patches in reverse Cuthill-McKee order): from a shuffled mesh the
    mean index distance of neighbours falls below the mesher's own order's and
    the largest one far below the shuffled order's."""
    from eulersr_b200.solver import DeviceMesh
    rng = np.random.default_rng(0)
    shuffled = diamond02.renumbered(rng.permutation(diamond02.n_cells))

    def dist(m, perm=None):
        inv = np.arange(m.n_cells)
        if perm is not None:
            inv = np.empty_like(perm)
            inv[perm] = np.arange(len(perm))
        c, k = np.nonzero(m.neighbors >= 0)
        return np.abs(inv[c] - inv[m.neighbors[c, k]])
    perm = DeviceMesh(shuffled).permutation()
    assert np.array_equal(np.sort(perm), np.arange(diamond02.n_cells))
    assert dist(shuffled, perm).mean() <= dist(diamond02).mean()
    assert dist(shuffled, perm).max() < dist(shuffled).max() / 4


@pytest.mark.parametrize("geom", ["naca0012", "diamond"])
def test_patches_cover_the_mesh_compactly(geom):
    """Patches of the renumbering: consecutive new cells, at most 24 each,
    covering the mesh; on the HR meshes about 72 % of the interior faces join
    two cells of one patch (K2 by patches evaluates those once), against
    under a fifth for blocks of 32 cells in plain RCM order."""
    from eulersr_b200.meshing.generate import cached_mesh
    from eulersr_b200.solver import DeviceMesh
    mesh = cached_mesh(geom, 0.025)
    dm = DeviceMesh(mesh)
    start = dm.patches()
    sizes = np.diff(start)
    assert start[0] == 0 and start[-1] == mesh.n_cells and sizes.min() >= 1 and sizes.max() <= 24
    assert np.mean(sizes == 24) > 0.95
    perm = dm.permutation()
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    patch_of = np.repeat(np.arange(len(sizes)), sizes)
    c, k = np.nonzero(mesh.neighbors >= 0)
    a, b = inv[c], inv[mesh.neighbors[c, k]]
    inner = np.mean(patch_of[a] == patch_of[b])
    assert inner > 0.7, inner
    dm.close()


def test_ctypes_structs_match_the_header(tmp_path):
    """Every ctypes mirror in _ffi.py has the size and field offsets the C
    compiler gives the header's struct (so a field added on one side only is
    caught without a GPU)."""
    import shutil
    import subprocess
    from pathlib import Path
    from eulersr_b200 import _ffi as F
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    pairs = {"esr_mesh_desc": F.MeshDesc, "esr_mesh_info": F.MeshInfo, "esr_params": F.Params,
             "esr_case": F.Case, "esr_result": F.Result, "esr_kernel_times": F.KernelTimes,
             "esr_tuning": F.Tuning, "esr_tuning_variant": F.TuningVariant}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "eulersr.h"', 'int main(void) {']
    for cname, py in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    inc = Path(__file__).resolve().parents[1] / "include"
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(inc), str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            parts = line.split()
            got[(parts[0], parts[1])] = int(parts[2])
    for cname, py in pairs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_ctypes_signatures_match_header_prototypes():
    """Every function the ctypes layer binds takes as many arguments as its
    prototype in include/eulersr.h, and every prototype has a binding."""
    import re
    from eulersr_b200 import _ffi as F
    txt = re.sub(r"/\*.*?\*/", "", F.HEADER.read_text(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(esr_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S):
        params = " ".join(m.group(2).split())
        protos[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    assert len(protos) >= 25
    missing = sorted(set(protos) - set(F._SIGS))
    assert not missing, missing
    for name, (_, args) in F._SIGS.items():
        assert name in protos, name
        assert len(args) == protos[name], (name, len(args), protos[name])


def test_no_cpu_fallback(diamond02):
    """The product path has no CPU fallback: on a machine without a usable GPU
    the solver fails with ESR_ERR_CUDA and the CUDA error text, and the warm
    start wrappers refuse host tensors and host devices before any launch."""
    import torch
    from eulersr_b200 import _ffi as F
    from eulersr_b200.solver import Solver
    from eulersr_b200.warmstart import mlp as mlp_mod, pipeline
    if not torch.cuda.is_available():
        with pytest.raises(F.EsrError) as e:
            Solver(diamond02, 2, precision="f32")
        assert e.value.code == F.ESR_ERR_CUDA
        assert "cuda" in str(e.value).lower()
    for wrap in (mlp_mod._p, pipeline._p):
        assert wrap(None) is None
        with pytest.raises(ValueError, match="CUDA tensor"):
            wrap(torch.zeros(4))
    with pytest.raises(ValueError, match="CUDA device"):
        mlp_mod.MLP(device="cpu")
    with pytest.raises(ValueError, match="CUDA device"):
        pipeline.WarmStart(None, device="cpu")


def _single_triangle(points=((0.0, 0.0), (1.0, 0.0), (0.0, 1.0)), markers=(3, 4, 2)):
    from eulersr_b200.mesh import Mesh
    return Mesh.from_arrays(np.array(points), [[0, 1, 2]], [[-1, -1, -1]], [[0, 1], [1, 2], [2, 0]], list(markers),
                            [[0, 1, 2]], dict(case="diamond"))


def test_mesh_edge_cases(diamond02):
    """Smallest and malformed meshes: one triangle whose three faces are all
    boundary faces prepares; an empty mesh, a degenerate triangle, an
    interior marker on a boundary edge and a neighbour that does not share
    the face are argument errors on the host, as are null arguments."""
    from eulersr_b200 import _ffi as F
    from eulersr_b200.mesh import Mesh
    from eulersr_b200.solver import DeviceMesh
    one = DeviceMesh(_single_triangle())
    assert one.n_cells == 1 and one.info.n_boundary_slots == 3 and one.info.n_wall_faces == 1
    assert list(one.permutation()) == [0]

    def rejects(mesh, text):
        with pytest.raises(F.EsrError) as e:
            DeviceMesh(mesh)
        assert e.value.code == F.ESR_ERR_ARG and text in str(e.value), str(e.value)

    rejects(_single_triangle(points=((0.0, 0.0), (1.0, 0.0), (2.0, 0.0))), "degenerate")
    rejects(_single_triangle(markers=(0, 4, 2)), "interior face marker")
    empty = Mesh.__new__(Mesh)
    empty.__dict__.update(diamond02.__dict__)
    empty.tris = np.zeros((0, 3), np.int32)
    empty.neighbors = np.zeros((0, 3), np.int32)
    empty.face_connectivity = np.zeros((0, 3), np.int32)
    rejects(empty, "empty mesh")
    # a neighbour that exists but does not list the shared face
    nb = diamond02.neighbors.copy()
    c = int(np.argmax((nb >= 0).all(axis=1)))
    far = next(j for j in range(diamond02.n_cells) if j != c and j not in set(nb[c].tolist())
               and c not in set(nb[j].tolist()))
    nb[c, 0] = far
    bad = Mesh.__new__(Mesh)
    bad.__dict__.update(diamond02.__dict__)
    bad.neighbors = nb
    rejects(bad, "does not list the shared face")
    L = F.lib()
    assert L.esr_mesh_create(None, None) == F.ESR_ERR_ARG
    assert b"null" in L.esr_last_error()


@pytest.mark.parametrize("field,value,text", [("precision", 2, "unknown precision"), ("flux", 7, "Unknown flux type"),
                                              ("reconstruction", 5, "Unknown reconstruction scheme"),
                                              ("time_scheme", 3, "unknown time scheme"), ("dt_mode", -1, "unknown dt mode"),
                                              ("stop_rule", 3, "unknown stop rule"), ("gamma", 1.0, "gamma must be > 1"),
                                              ("slots", 0, "slots_per_mesh must be > 0")])
def test_solver_create_checks_arguments_first(diamond02, field, value, text):
    """esr_solver_create checks every argument before it touches a device, so
    a bad one is ESR_ERR_ARG with the reference's message on any machine."""
    from eulersr_b200 import _ffi as F
    from eulersr_b200.solver import DeviceMesh
    L = F.lib()
    dm = DeviceMesh(diamond02)
    p = F.Params(precision=0, flux=0, reconstruction=0, time_scheme=0, dt_mode=0, stop_rule=0, gamma=1.4,
                 threshold=1e-6, check_every=10, patience=3, device=0, use_graphs=1, block_size=0)
    slots = (C.c_int32 * 1)(4)
    if field == "slots":
        slots[0] = value
    else:
        setattr(p, field, value)
    meshes = (C.c_void_p * 1)(dm.handle.value)
    h = C.c_void_p()
    assert L.esr_solver_create(meshes, slots, 1, C.byref(p), C.byref(h)) == F.ESR_ERR_ARG
    assert text in L.esr_last_error().decode()
    assert not h.value
    assert L.esr_solver_create(None, slots, 1, C.byref(p), C.byref(h)) == F.ESR_ERR_ARG


def test_item_divider_is_exact(tmp_path):
    """The divide-free n / d of the step kernels' item mapping (esr_layout.h:
    make_divider / divide, also what compaction sets for the live slots) is
    exact for every d up to 4096 on edge and random n below 2^31."""
    import shutil
    import subprocess
    from pathlib import Path
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "div.cpp"
    src.write_text('''
#include <cstdio>
#include <random>
#include "esr_layout.h"
using namespace esr;
int main() {
  std::mt19937_64 rng(7);
  long bad = 0;
  for (unsigned d = 1; d <= 4096; ++d) {
    const Divider v = make_divider(d);
    const unsigned top = 2147483647u;
    unsigned ns[6] = {0u, d - 1, d, top, top - top % d, top - top % d - 1};
    for (unsigned n : ns) bad += divide(n, v) != n / d;
    for (int i = 0; i < 2000; ++i) { unsigned n = (unsigned)(rng() % 2147483648ull); bad += divide(n, v) != n / d; }
  }
  std::printf("%ld\\n", bad);
  return bad != 0;
}
''')
    exe = tmp_path / "div"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", str(root / "eulersr_b200" / "csrc"), str(src), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "0", r.stdout
