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


@pytest.mark.parametrize("mach,aoa", [(2.0, 0.0), (2.5, 3.0)])
def test_theory_forces_on_mesh_equal_analytic(mach, aoa):
    """The theory's face pressures placed on the wall cells and integrated by
    the force routine give the analytic shock-expansion CD and CL (the body's
    faces are exact segments of the four panels)."""
    from conftest import load_mesh
    from eulersr_b200.postproc import diamond_theory
    from eulersr_b200 import theory_validation as TV
    m = load_mesh("diamond_h0.1")
    cx, cy = m.metadata["center"]["cx"], m.metadata["center"]["cy"]
    panels = TV.diamond_panels(mach, aoa, 5.0)
    assert TV.all_attached(panels)
    cd, cl = TV.theory_forces(m, panels, mach, cx, cy)
    th = diamond_theory(mach, aoa, 5.0)
    assert cd == pytest.approx(th.cd, rel=1e-9)
    assert cl == pytest.approx(th.cl, rel=1e-9, abs=1e-12)
    for n in TV.PANEL_NAMES:
        assert panels[n].p_ratio_freestream == pytest.approx(th.p_faces[n], rel=1e-12)
    # M=1.05 detaches the front shocks: the campaigns skip such points
    assert not TV.all_attached(TV.diamond_panels(1.05, 0.0, 5.0))


def test_measure_shock_angle_on_a_ridge():
    """Cells whose |grad p| peaks along a line through the leading edge at
    angle beta give back beta."""
    from eulersr_b200 import theory_validation as TV
    rng = np.random.default_rng(4)
    cx, cy, chord, height = 1.5, 2.0, 1.0, math.tan(math.radians(5.0))
    x_le = cx - 0.5 * chord
    pts = np.column_stack([rng.uniform(x_le - 0.35, x_le + 0.45, 20000), rng.uniform(cy - 0.3, cy + 0.3, 20000)])
    beta = math.radians(41.0)
    for side, sgn in (("upper", 1.0), ("lower", -1.0)):
        d = np.abs(np.sin(beta) * (pts[:, 0] - x_le) - np.cos(beta) * sgn * (pts[:, 1] - cy))
        grad = np.column_stack([np.exp(-(d / 0.004) ** 2), np.zeros(len(pts))])
        got = TV.measure_shock_angle(pts, grad, cx, cy, chord, height, 0.0, side)
        assert got == pytest.approx(41.0, abs=0.3)
    assert TV.measure_shock_angle(pts[:5], grad[:5], cx, cy, chord, height, 0.0, "upper") is None


def test_theory_campaigns_on_bundles(tmp_path):
    """Both campaigns over bundles laid out as the grid driver writes them: a
    field that carries the theory's pressures on the wall cells has zero CD,
    CL and plateau-Cp error; the CSVs have the reference's columns."""
    from eulersr_b200.mesh import Mesh
    from eulersr_b200.meshing import generate as G
    from eulersr_b200 import mesh_convergence as MC
    from eulersr_b200 import theory_validation as TV
    mesh_dir, raw_dir = tmp_path / "meshes", tmp_path / "raw"
    mach, aoa = 2.0, 0.0
    chain = [0.2, 0.15]       # coarser levels have under 3 faces per panel: no plateau
    for h in chain:
        G.generate("diamond", h, mesh_dir)
        m = Mesh.load(G.mesh_path(mesh_dir, "diamond", h))
        cx, cy = m.metadata["center"]["cx"], m.metadata["center"]["cy"]
        panels = TV.diamond_panels(mach, aoa, 5.0)
        p = np.ones(m.n_cells)
        first = TV._first_owner(m)
        mid = m.face_midpoints()
        for f in np.nonzero(m.face_markers == m.force_marker())[0]:
            p[first[f] // 3] = panels[TV.panel_of(mid[f, 0], mid[f, 1], cx, cy)].p_ratio_freestream
        W = np.zeros((m.n_cells, 4))
        W[:, 0] = 1.0
        W[:, 3] = p / 0.4
        grad = np.zeros((m.n_cells, 4, 2))
        d = raw_dir / MC.format_h(h) / "AOA0.00"
        d.mkdir(parents=True)
        np.savez(d / "AOA0.00_M2.00_HLLC_MUSCL_SRK2_t3.00.npz", conservatives=W, node_pos=m.barycenter,
                 primitives_grad=grad)
    pts = [("P6_mach2_symetrique", mach, aoa), ("P2_supersonique_marginal", 1.05, 0.0)]
    path = TV.run_theory_validation(raw_dir, mesh_dir, tmp_path / "theory", points=pts, h=0.2)
    lines = path.read_text().splitlines()
    assert lines[0].startswith("label,mach,aoa,Cd_fvm,Cd_theory")
    assert len(lines) == 1 + 4                      # the detached point is skipped
    for line in lines[1:]:
        f = line.split(",")
        assert float(f[3]) == pytest.approx(float(f[4]), abs=1e-6)    # CD
        assert float(f[8]) == pytest.approx(float(f[9]), abs=1e-6)    # plateau Cp
    errs, fit = TV.run_wall_convergence(raw_dir, mesh_dir, tmp_path / "wall", points=pts, h_all=chain)
    rows = errs.read_text().splitlines()
    assert len(rows) == 1 + len(chain)
    for line in rows[1:]:
        f = line.split(",")
        assert float(f[7]) < 1e-9 and float(f[10]) < 1e-9 and float(f[11]) < 1e-9
    assert fit.read_text().splitlines() == ["label,mach,aoa,quantity,p_order,r2,n_points"]


def test_fit_order():
    from eulersr_b200.theory_validation import fit_order
    rows = [dict(h=h, e=3.0 * h ** 1.5) for h in (0.1, 0.05, 0.025, 0.0125, 0.2)]
    p, r2, n = fit_order(rows, "e")
    assert n == 4 and p == pytest.approx(1.5, abs=1e-10) and r2 == pytest.approx(1.0, abs=1e-12)
    assert fit_order(rows[:2], "e")[0] is None


def test_loss_weights_formula():
    """Shock weights of the training rows (preprocessing/dataset.py:168-170):
    1 + |grad p| / mean |grad p|, capped at 5."""
    from eulersr_b200.warmstart.pipeline import loss_weights
    g = np.array([[0.0, 0.0], [0.0, 0.0], [0.0, 0.0], [3.0, 4.0], [0.0, 1.0], [60.0, 80.0]], np.float32)
    gp = np.array([0.0, 0.0, 0.0, 5.0, 1.0, 100.0])
    want = np.minimum(1.0 + gp / gp.mean(), 5.0)
    assert np.allclose(loss_weights(g), want, rtol=1e-6)
    assert loss_weights(g).dtype == np.float32 and loss_weights(g).max() == 5.0
    assert np.allclose(loss_weights(g, factor=0.0), 1.0)


def test_wall_features_distance_and_normal():
    """Distance to the nearest of 8 samples per wall face and the face normal
    turned towards the query point (utils/aero.py:154-177), on the diamond."""
    from conftest import load_mesh
    from eulersr_b200.warmstart.features import wall_features
    m = load_mesh("diamond_h0.1")
    cx, cy = m.metadata["center"]["cx"], m.metadata["center"]["cy"]
    chord, height = m.metadata["chord"], m.metadata["height"]
    x_le, top = cx - chord / 2, cy + height / 2
    eps = math.atan(height / chord)
    # the upper-front face's outward normal and a point 0.1 off its middle
    n_uf = np.array([-math.sin(eps), math.cos(eps)])
    mid_uf = np.array([x_le + chord / 4, cy + height / 4])
    q = np.array([[cx, top + 0.3], [x_le - 0.2, cy], mid_uf + 0.1 * n_uf, mid_uf - 0.005 * n_uf])
    d, n = wall_features(m, q)
    assert d[0] == pytest.approx(0.3, abs=1e-12) and n[0, 1] > 0.99   # the top vertex is a sample
    assert d[1] == pytest.approx(0.2, abs=1e-12) and n[1, 0] < 0      # the leading edge is a sample
    faces = m.faces[m.face_markers == m.force_marker()]
    seg = np.linalg.norm(m.points[faces[:, 1]] - m.points[faces[:, 0]], axis=1).max()
    assert 0.1 - 1e-12 <= d[2] <= math.hypot(0.1, seg / 14) + 1e-12     # samples 1/7 of a face apart
    assert n[2] @ n_uf == pytest.approx(1.0, abs=1e-9)
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0)
    assert n[3] @ n_uf == pytest.approx(-1.0, abs=1e-9)               # turned towards a point inside


def test_gas_dynamics_textbook_values():
    """Prandtl-Meyer angles and the M=2, 10-degree oblique shock and
    expansion against the standard tables (gamma 1.4)."""
    from eulersr_b200.postproc import expansion, oblique_shock, prandtl_meyer
    for M, nu in ((1.5, 11.91), (2.0, 26.38), (3.0, 49.76)):
        assert math.degrees(prandtl_meyer(M)) == pytest.approx(nu, abs=0.01)
    beta, M2, pr = oblique_shock(2.0, math.radians(10.0))
    assert math.degrees(beta) == pytest.approx(39.31, abs=0.01)
    assert M2 == pytest.approx(1.64, abs=0.005) and pr == pytest.approx(1.7066, abs=1e-4)
    M2e, pre = expansion(2.0, math.radians(10.0))
    assert math.degrees(prandtl_meyer(M2e)) == pytest.approx(36.38, abs=0.01)
    assert M2e == pytest.approx(2.385, abs=0.002)
    # isentropic: p2/p1 from the stagnation-pressure ratio of the two Mach numbers
    assert pre == pytest.approx(((1 + 0.2 * 4.0) / (1 + 0.2 * M2e ** 2)) ** 3.5, rel=1e-12)
