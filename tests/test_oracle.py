"""Known-answer properties of the oracle (CPU only).

The reference has no tests or golden vectors and JAX is absent here; the
oracle is pinned bit for bit to the reference's own solver source run with
NumPy (tests/test_reference_fixtures.py), and these tests add properties
every correct implementation of euler_solver.py / helper.py satisfies, plus a
committed regression fixture of the oracle itself.
"""
import numpy as np
import pytest

from conftest import oracle_mesh, rel_err
from oracle import euler_oracle as O


def _box_mesh():
    """Body-free box: freestream must be preserved exactly (up to rounding)."""
    from eulersr_b200.mesh import Mesh
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(0)
    g = np.linspace(0, 1, 9)
    X, Y = np.meshgrid(g, g)
    pts = np.column_stack([X.ravel(), Y.ravel()])
    inner = (pts[:, 0] > 0) & (pts[:, 0] < 1) & (pts[:, 1] > 0) & (pts[:, 1] < 1)
    pts[inner] += 0.02 * rng.standard_normal((inner.sum(), 2))
    tri = Delaunay(pts)
    return Mesh.from_triangles(pts, tri.simplices, box=(0, 1, 0, 1), metadata={'case': 'box'})


def test_freestream_preserved_without_body():
    m = _box_mesh()
    for dt_ in (np.float64, np.float32):
        om = oracle_mesh(m, dt_)
        W, inlet = O.initialize(m.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.0, aoa=3.0,
                                                case='diamond'), dt_)
        R = O.residual(W, om, inlet)
        scale = np.abs(O.get_flux(*O.build_reconstruction(W, om, inlet=inlet), om.normals,
                                  om.surface[om.face_connectivity]) * 0 + 10.0)
        assert np.max(np.abs(R)) <= (1e-12 if dt_ == np.float64 else 2e-4) * scale.max()


def _states(n, seed):
    rng = np.random.default_rng(seed)
    P = np.column_stack([rng.uniform(0.5, 2.0, n), rng.uniform(-2, 3, n), rng.uniform(-1, 1, n),
                         rng.uniform(0.3, 3.0, n)])
    return O.get_conserved(P)


def test_hllc_consistency():
    """F(U, U, n) equals the physical flux."""
    W = _states(200, 1)
    rng = np.random.default_rng(2)
    th = rng.uniform(0, 2 * np.pi, 200)
    n = np.column_stack([np.cos(th), np.sin(th)])
    F = O.get_flux(W[:, None, :], W[:, None, :], n[:, None, :], np.ones((200, 1)))
    P = O.get_primitive(W)
    un = P[:, 1] * n[:, 0] + P[:, 2] * n[:, 1]
    Fp = np.column_stack([P[:, 0] * un, P[:, 0] * P[:, 1] * un + P[:, 3] * n[:, 0],
                          P[:, 0] * P[:, 2] * un + P[:, 3] * n[:, 1], (W[:, 3] + P[:, 3]) * un])
    assert np.allclose(F, Fp, rtol=1e-12, atol=1e-12)


def test_hllc_antisymmetry_and_rotation():
    WL, WR = _states(300, 3), _states(300, 4)
    rng = np.random.default_rng(5)
    th = rng.uniform(0, 2 * np.pi, 300)
    n = np.column_stack([np.cos(th), np.sin(th)])
    one = np.ones((300, 1))
    F = O.get_flux(WL[:, None], WR[:, None], n[:, None], one)
    Fr = O.get_flux(WR[:, None], WL[:, None], -n[:, None], one)
    assert np.allclose(F, -Fr, rtol=1e-10, atol=1e-10)
    # rotation invariance: rotate states and normal by the same angle
    a = 0.7
    Rm = np.array([[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]])
    def rot(W):
        W = W.copy()
        W[:, 1:3] = W[:, 1:3] @ Rm.T
        return W
    F2 = O.get_flux(rot(WL)[:, None], rot(WR)[:, None], (n @ Rm.T)[:, None], one)
    F2[:, 1:3] = F2[:, 1:3] @ Rm
    assert np.allclose(F, F2, rtol=1e-9, atol=1e-9)


def test_lsq_exact_on_linear_fields(diamond02):
    om = oracle_mesh(diamond02, np.float64)
    a = np.array([0.3, -1.2, 0.5, 2.0]); bx = np.array([0.1, 0.4, -0.2, 0.7]); by = np.array([-0.3, 0.2, 0.9, 0.1])
    x, y = om.barycenter[:, 0], om.barycenter[:, 1]
    P = a + bx * x[:, None] + by * y[:, None]
    PL = np.repeat(P[:, None], 3, axis=1)
    PR = P[diamond02.neighbors]
    interior = np.all(diamond02.neighbors >= 0, axis=1)
    g = O.lsq_gradient(PL, PR, om)
    assert np.allclose(g[interior, :, 0], bx, atol=1e-10)
    assert np.allclose(g[interior, :, 1], by, atol=1e-10)


def test_limiter_range(diamond02):
    om = oracle_mesh(diamond02, np.float64)
    W0, inlet = O.initialize(diamond02.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0,
                                                     case='diamond'))
    rng = np.random.default_rng(0)
    P0 = O.get_primitive(W0) * (1 + 0.1 * rng.standard_normal(W0.shape))
    W = O.get_conserved(P0)
    WL = np.repeat(W[:, None], 3, axis=1)
    WR = O.bc_state(W[diamond02.neighbors], WL, om, inlet)
    PL, PR = O.get_primitive(WL), O.get_primitive(WR)
    phi = O.limiter(PL, PR, O.lsq_gradient(PL, PR, om), om)
    # Venkatakrishnan with K=0: phi in [0, (y^2+2y)/(y^2+y+2) max ~ 1.0937]
    assert phi.min() >= -1e-12 and phi.max() <= 1.094


def test_venkat_maximum():
    # with K=0, f(y) = (y^2 + 2y) / (y^2 + y + 2) for y = a/b peaks at y* = 2 + 2 sqrt(2)
    y = np.linspace(0.01, 50, 100000)
    f = O.venkatakrishnan(y, np.ones_like(y))
    ys = 2 + 2 * np.sqrt(2)
    assert abs(f.max() - (ys ** 2 + 2 * ys) / (ys ** 2 + ys + 2)) < 1e-6


def test_golden_regression(diamond02, golden):
    g = np.load(golden / "oracle_diamond_h0.2_M2.5_a5_srk2x20.npz")
    om = oracle_mesh(diamond02, np.float64)
    W, inlet = O.initialize(diamond02.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0,
                                                    case='diamond'))
    dt = O.get_dt(W, om, CFL=0.6)
    assert dt == pytest.approx(float(g['dt']), rel=1e-15)
    for _ in range(int(g['steps'])):
        W = O.time_step_srk2(W, om, dt, inlet)
    assert rel_err(W, g['W']) <= 1e-13


def test_stop_rule_semantics(diamond02):
    """euler/main.py:147-158: a patience-2 streak stops at the streak start."""
    om = oracle_mesh(diamond02, np.float64)
    cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0, case='diamond', CFL=0.6, tf=2.0,
               stationarity_threshold=5e-4, stationarity_check_every=20, stationarity_patience=2)
    W, inlet = O.initialize(diamond02.n_cells, cfg)
    r = O.run(W, om, inlet, cfg)
    if r.converged:
        steps = [s for s, rel in r.rel_history]
        rels = [rel for s, rel in r.rel_history]
        assert rels[-1] <= 5e-4 and rels[-2] <= 5e-4
        assert r.stopping_step == steps[-2]
    assert r.n_max == int(2.0 / r.dt) + 1


def test_transonic_cfl_clamp(naca02):
    om = oracle_mesh(naca02, np.float64)
    cfg = dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=0.8, aoa=0.0, case='naca0012', CFL=0.6, tf=0.01,
               stationarity_threshold=1e-30, stationarity_check_every=5)
    W, inlet = O.initialize(naca02.n_cells, cfg)
    r = O.run(W, om, inlet, cfg)
    assert r.dt == pytest.approx(float(O.get_dt(W, om, CFL=0.45)), rel=1e-15)


def test_idw_weights_normalised():
    rng = np.random.default_rng(0)
    d = rng.uniform(0.01, 1, (50, 6))
    w = O.idw_weights(d)
    assert np.allclose(w.sum(1), 1.0)
    src = rng.standard_normal((40, 4)).astype(np.float32)
    idx = rng.integers(0, 40, (50, 6))
    out = O.idw_predict(src, idx, d)
    assert out.shape == (50, 4) and out.dtype == np.float32


def test_c_port_matches_numpy_oracle(diamond02):
    """The multi-threaded C restatement (CPU baseline) agrees with the NumPy oracle."""
    from oracle.cport import CpuCase
    cc = CpuCase(diamond02, 2.5, 5.0, np.float64)
    Wc = cc.srk2(cc.W0, 20)
    om = cc.om
    W = cc.W0
    for _ in range(20):
        W = O.time_step_srk2(W, om, cc.dt, cc.inlet)
    assert rel_err(Wc, W) <= 1e-12
    c32 = CpuCase(diamond02, 2.5, 5.0, np.float32)
    assert rel_err(c32.srk2(c32.W0, 20), W) <= 1e-5


def test_c_port_local_dt_matches_numpy_oracle(diamond02):
    """The C restatement's local-CFL SRK2 (the converged-cases CPU baseline
    runs it) agrees with the oracle's time_step_srk2_local."""
    from oracle.cport import CpuCase
    cc = CpuCase(diamond02, 0.85, 2.0, np.float64)
    Wc = cc.srk2_local(cc.W0, 20, 0.45)
    W = cc.W0
    for _ in range(20):
        W = O.time_step_srk2_local(W, cc.om, 0.45, cc.inlet)
    assert rel_err(Wc, W) <= 1e-12


def test_rusanov_consistency_and_antisymmetry():
    """The Rusanov branch of getFlux: F(U, U, n) is the physical flux and
    F(L, R, n) = -F(R, L, -n)."""
    W = _states(200, 11)
    rng = np.random.default_rng(12)
    th = rng.uniform(0, 2 * np.pi, 200)
    n = np.column_stack([np.cos(th), np.sin(th)])
    one = np.ones((200, 1))
    F = O.get_flux(W[:, None], W[:, None], n[:, None], one, flux='rusanov')
    H = O.get_flux(W[:, None], W[:, None], n[:, None], one, flux='hllc')
    assert np.allclose(F, H, rtol=1e-12, atol=1e-12)
    WR = _states(200, 13)
    Fa = O.get_flux(W[:, None], WR[:, None], n[:, None], one, flux='rusanov')
    Fb = O.get_flux(WR[:, None], W[:, None], -n[:, None], one, flux='rusanov')
    assert np.allclose(Fa, -Fb, rtol=1e-10, atol=1e-10)


def test_slip_wall_ghost_reflects_the_normal_velocity(diamond02):
    """helper.py:196-204: at a wall slot the ghost keeps density, pressure and
    tangential velocity and reverses the normal velocity."""
    om = oracle_mesh(diamond02, np.float64)
    n = diamond02.n_cells
    W = np.repeat(_states(n, 21)[:, None, :], 3, axis=1)
    G = O.bc_state(W.copy(), W, om, inlet=O.get_conserved(np.array([1.0, 2.0, 0.0, 1.0])))
    wall = diamond02.face_markers[diamond02.face_connectivity] == 2
    assert wall.sum() > 10
    P, Pg = O.get_primitive(W[wall]), O.get_primitive(G[wall])
    nrm = om.normals[wall]
    un, ung = (P[:, 1:3] * nrm).sum(1), (Pg[:, 1:3] * nrm).sum(1)
    t = np.column_stack([-nrm[:, 1], nrm[:, 0]])
    assert np.allclose(ung, -un, atol=1e-12)
    assert np.allclose((Pg[:, 1:3] * t).sum(1), (P[:, 1:3] * t).sum(1), atol=1e-12)
    assert np.allclose(Pg[:, [0, 3]], P[:, [0, 3]], rtol=1e-12)
    # inflow slots take the inlet state, outflow slots copy the cell
    mk = diamond02.face_markers[diamond02.face_connectivity]
    assert np.allclose(G[mk == 3], O.get_conserved(np.array([1.0, 2.0, 0.0, 1.0])))
    assert np.array_equal(G[mk == 4], W[mk == 4])


def test_sponge_vanishes_at_freestream_and_in_the_core(diamond02):
    """helper.py:262-295: sigma >= 0 and zero outside the bands of 0.2 Ly along
    the top and bottom; the source is zero where the state is the inlet's."""
    om = oracle_mesh(diamond02, np.float64)
    W, inlet = O.initialize(diamond02.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.0, aoa=0.0,
                                                    case='diamond'), np.float64)
    assert np.abs(O.sponge_source(W, om, inlet)).max() == 0.0
    Wp = W * 1.1
    S = O.sponge_source(Wp, om, inlet)
    y = om.barycenter[:, 1]
    y0, y1 = om.points[:, 1].min(), om.points[:, 1].max()
    core = np.minimum(y - y0, y1 - y) >= 0.2 * (y1 - y0)
    assert np.abs(S[core]).max() == 0.0
    sigma = S[:, 0] / (inlet[0] - Wp[:, 0])
    assert (sigma >= 0).all() and sigma.max() > 0


def test_global_dt_is_the_minimum_local_dt(diamond02):
    om = oracle_mesh(diamond02, np.float64)
    W = _states(diamond02.n_cells, 31)
    assert O.get_dt(W, om, CFL=0.6) == O.get_local_dt(W, om, CFL=0.6).min()


def test_every_time_scheme_preserves_freestream_without_body():
    m = _box_mesh()
    om = oracle_mesh(m, np.float64)
    W, inlet = O.initialize(m.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=1.5, aoa=10.0,
                                            case='diamond'), np.float64)
    dt = O.get_dt(W, om, CFL=0.5)
    for name, fn in O.TIME_SCHEMES.items():
        Wn = fn(W, om, dt, inlet)
        assert np.allclose(Wn, W, rtol=0, atol=1e-12), name


def test_mlp_oracle_gradients_match_finite_differences():
    """The MLP oracle's exact (float64) backward against central differences
    of its loss, on sampled weights and biases of every layer: the oracle the
    BF16 GPU gradients are held to is itself right."""
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(7)
    P = {"W0": rng.standard_normal((256, 128)) * 0.1, "b0": rng.standard_normal(256) * 0.1}
    for l in (1, 2, 3):
        P[f"W{l}"] = rng.standard_normal((256, 256)) * 0.06
        P[f"b{l}"] = rng.standard_normal(256) * 0.1
    P["W4"], P["b4"] = rng.standard_normal((4, 256)) * 0.1, rng.standard_normal(4) * 0.1
    X = np.zeros((16, 128))
    X[:, :13] = rng.standard_normal((16, 13))
    base, tgt = rng.standard_normal((16, 4)), rng.standard_normal((16, 4))
    w, inv_den = 1 + 4 * rng.random(16), np.array([1.3, 0.7, 2.0, 1.1])

    def loss(params):
        y, _ = MO.forward(params, X, base, bf16=False)
        return MO.loss_and_grad(y, tgt, w, inv_den)[0]

    y, acts = MO.forward(P, X, base, bf16=False)
    _, dy = MO.loss_and_grad(y, tgt, w, inv_den)
    g = MO.backward(P, acts, dy, bf16=False)
    h = 1e-6
    for k in ("W0", "b0", "W1", "b2", "W3", "b3", "W4", "b4"):
        for _ in range(4):
            idx = tuple(rng.integers(0, s) for s in P[k].shape)
            Pp = {kk: v.copy() for kk, v in P.items()}
            Pm = {kk: v.copy() for kk, v in P.items()}
            Pp[k][idx] += h
            Pm[k][idx] -= h
            fd = (loss(Pp) - loss(Pm)) / (2 * h)
            assert abs(fd - g[k][idx]) <= 1e-6 * max(1e-3, abs(fd)), (k, idx, fd, g[k][idx])


def test_mlp_loss_is_the_shock_weighted_relative_mse():
    """With the batch's own denominators, the oracle's loss is loss.py:20-23's
    shock_weighted_rel_mse: mean over variables of
    mean_rows(w (pred - target)^2) / (mean_rows(target^2) + 1e-8)."""
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(9)
    y, t = rng.standard_normal((50, 4)), rng.standard_normal((50, 4)) * [1.0, 2.0, 0.5, 3.0]
    w = 1 + 4 * rng.random(50)
    ref = ((w[:, None] * (y - t) ** 2).mean(0) / ((t ** 2).mean(0) + 1e-8)).mean()
    L, _ = MO.loss_and_grad(y, t, w, 1.0 / ((t ** 2).mean(0) + 1e-8))
    assert L == pytest.approx(ref, rel=1e-13)
