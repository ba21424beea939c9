"""Post-processing on solver outputs (CPU only): host force coefficients and
wall profile, Richardson/GCI, and the mesh-convergence campaign over bundles
laid out as the grid driver writes them."""
import math

import numpy as np
import pytest

from conftest import oracle_mesh


def _field(mesh, mach, seed=0):
    """A smooth non-uniform conserved field around the freestream of ``mach``."""
    from eulersr_b200.solver import freestream
    W = np.tile(freestream(mach, 0.0, dtype=np.float64), (mesh.n_cells, 1))
    x, y = mesh.barycenter.T
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.05, 0.1, 4)
    W *= 1.0 + a[None, :] * np.sin(1.3 * x + 0.7 * y)[:, None]
    return W


def test_force_coefficients_match_oracle(diamond02):
    from eulersr_b200.postproc import force_coefficients
    from oracle import euler_oracle as O
    W = _field(diamond02, 2.0)
    om = oracle_mesh(diamond02, np.float64)
    cd_o, cl_o = O.force_coefficients(W, om, 1.0, 2.0 * math.sqrt(1.4), 1.0)
    cd, cl = force_coefficients(diamond02, W, 2.0)
    assert cd == pytest.approx(cd_o, rel=1e-12, abs=1e-14)
    assert cl == pytest.approx(cl_o, rel=1e-12, abs=1e-14)
    # a uniform pressure exerts no net force on a closed body
    from eulersr_b200.solver import freestream
    cd0, cl0 = force_coefficients(diamond02, np.tile(freestream(2.0, 0.0, dtype=np.float64), (diamond02.n_cells, 1)), 2.0)
    assert abs(cd0) < 1e-12 and abs(cl0) < 1e-12


def test_wall_profile(diamond02):
    from eulersr_b200.postproc import wall_profile
    from eulersr_b200.solver import freestream
    W = np.tile(freestream(1.7, 0.0, dtype=np.float64), (diamond02.n_cells, 1))
    prof = wall_profile(diamond02, W)
    n = prof["face_ids"].size
    assert n > 3
    assert np.all(np.isin(diamond02.face_markers[prof["face_ids"]], diamond02.wall_markers()))
    assert np.all(np.diff(prof["x"]) >= 0)          # sorted by midpoint x
    assert np.all(np.diff(prof["s"]) > 0) and prof["s"][0] == 0.0
    y_mid = 0.5 * (diamond02.points[:, 1].min() + diamond02.points[:, 1].max())
    assert np.all(prof["y"] <= y_mid + 1e-12)       # the lower surface
    assert np.allclose(prof["mach"], 1.7, rtol=1e-12)
    assert np.allclose(prof["pressure"], 1.0, rtol=1e-12)


def test_richardson_gci_known_order():
    from eulersr_b200.mesh_convergence import richardson_gci
    chain = [0.4, 0.2, 0.1, 0.05]
    vals = {h: 0.05 + 0.3 * h ** 2 for h in chain}
    out = richardson_gci(vals, chain)
    assert len(out) == 2
    for t in out:
        assert t["p_obs"] == pytest.approx(2.0, abs=1e-10)
        assert t["extrap"] == pytest.approx(0.05, abs=1e-12)
        f2, f3 = vals[t["h_mid"]], vals[t["h_fine"]]
        assert t["gci_fine_pct"] == pytest.approx(1.25 * abs((f3 - f2) / f3) / 3.0 * 100.0, rel=1e-10)
    # oscillating values: no order
    osc = {0.4: 1.0, 0.2: 1.1, 0.1: 1.0}
    assert richardson_gci(osc, [0.4, 0.2, 0.1])[0]["p_obs"] is None


def test_mesh_convergence_campaign(tmp_path):
    from eulersr_b200.mesh import Mesh
    from eulersr_b200.meshing import generate as G
    from eulersr_b200 import mesh_convergence as MC
    from eulersr_b200.postproc import force_coefficients
    mesh_dir, raw_dir, out_dir = tmp_path / "meshes", tmp_path / "raw", tmp_path / "out"
    chain = [0.4, 0.3, 0.2]
    cds = {}
    for h in chain:
        G.generate("diamond", h, mesh_dir)
        m = Mesh.load(G.mesh_path(mesh_dir, "diamond", h))
        W = _field(m, 1.5, seed=int(h * 10))
        d = raw_dir / MC.format_h(h) / "AOA0.00"
        d.mkdir(parents=True)
        # an older snapshot of the same case is ignored in favour of the latest
        np.savez(d / "AOA0.00_M1.50_HLLC_MUSCL_SRK2_t0.50.npz", conservatives=np.zeros_like(W))
        np.savez(d / "AOA0.00_M1.50_HLLC_MUSCL_SRK2_t2.00.npz", conservatives=W.astype(np.float32))
        cds[h] = force_coefficients(m, W.astype(np.float32), 1.5)[0]
    raw_csv, gci_csv = MC.campaign(raw_dir, mesh_dir, out_dir, points=[("P3", 1.5, 0.0)],
                                   h_all=chain, h_gci=[0.4, 0.2, 0.1])
    lines = raw_csv.read_text().splitlines()
    assert lines[0] == "label,mach,aoa,h,n_cells,cd,cl,wall_profile_rel_err"
    assert len(lines) == 1 + len(chain)
    for line in lines[1:]:
        f = line.split(",")
        assert float(f[5]) == pytest.approx(cds[float(f[3])], abs=2e-6)
    assert lines[-1].split(",")[-1] != ""          # finest level against itself: 0
    assert float(lines[-1].split(",")[-1]) == 0.0
    # the ratio-2 chain lacks h=0.1 here, so no GCI triplet
    assert gci_csv.read_text().splitlines() == ["label,mach,aoa,h_coarse,h_mid,h_fine,quantity,p_obs,extrap,gci_fine_pct"]
