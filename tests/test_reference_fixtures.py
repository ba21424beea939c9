"""The oracle and the package's host utilities against golden vectors made
by EulerSR's own NumPy code (tests/golden/make_reference_fixtures.py):
IDW weights (utils/metrics.py:9-14), wall distance and normal
(utils/aero.py:154-177) and the host CL/CD (utils/aero.py:85-110)."""
import numpy as np
import pytest

from conftest import GOLDEN, load_mesh


@pytest.fixture(scope="module")
def ref():
    return np.load(GOLDEN / "reference_utils.npz")


def test_idw_matches_reference_weights(ref):
    """The oracle's IDW weights equal the reference's, and its prediction is
    those weights (rounded to float32, as eval/core.py:135-142 applies them)
    on the neighbours' values; the GPU kernel is held to the oracle."""
    from oracle import euler_oracle as O
    dist, w = ref["idw_dist"], ref["idw_w"]
    assert np.allclose(O.idw_weights(dist), w, rtol=1e-14, atol=0)
    rng = np.random.default_rng(2)
    src = rng.standard_normal((400, 4)).astype(np.float32)
    idx = rng.integers(0, 400, dist.shape)
    got = O.idw_predict(src, idx, dist)
    want = (w.astype(np.float32)[:, :, None] * src[idx]).sum(axis=1)
    assert np.allclose(got, want, rtol=1e-6, atol=1e-6)


def test_wall_features_match_reference(ref):
    from eulersr_b200.warmstart.features import wall_features
    mesh = load_mesh("diamond_h0.2")
    d, n = wall_features(mesh, ref["wall_query"])
    assert np.allclose(d, ref["wall_dist"], rtol=0, atol=1e-12)
    assert np.allclose(n, ref["wall_normal"], rtol=0, atol=1e-9)


def test_host_force_coefficients_match_reference(ref):
    """postproc.force_coefficients against the reference's aero_coeffs, which
    rounds the wall normals and lengths to float32 (hence 1e-6)."""
    from eulersr_b200.postproc import force_coefficients
    mesh = load_mesh("diamond_h0.2")
    prim = ref["aero_prim"]
    r, u, v, p = prim.T
    W = np.stack([r, r * u, r * v, p / 0.4 + 0.5 * r * (u * u + v * v)], 1)
    cd, cl = force_coefficients(mesh, W, float(ref["aero_mach"]))
    assert cd == pytest.approx(float(ref["aero_cd"]), rel=1e-6, abs=1e-9)
    assert cl == pytest.approx(float(ref["aero_cl"]), rel=1e-6, abs=1e-9)


def test_graph_npz_matches_reference_export(ref):
    """Every array the reference's euler/graph.py export_graph wrote for the
    golden mesh (nodes, directed edges with their normals, lengths, vectors,
    face ids, boundary markers and kinds, boundary faces, inlet state,
    snapshots) is identical in the package's graph.npz."""
    mesh = load_mesh("diamond_h0.2")
    snap = ref["graph_snapshot"]
    ours = mesh.graph_arrays({0.5: snap, 1.25: 2 * snap}, [1.0, 2.0, 0.1, 4.5])
    theirs = np.load(GOLDEN / "reference_graph.npz")
    assert set(theirs.files) <= set(ours)
    for k in theirs.files:
        assert ours[k].dtype == theirs[k].dtype, k
        assert np.array_equal(ours[k], theirs[k]), k


def test_config_defaults_and_output_names_match_reference():
    """The default configuration (euler/config.toml through euler/config.py)
    and the output names the reference builds from a configuration: mesh-size
    tag, condition tag, snapshot name."""
    import json
    from eulersr_b200 import config as Cfg
    ref = json.loads((GOLDEN / "reference_config.json").read_text())
    ours = Cfg.load_default_config()
    for k, v in ref["default"].items():
        assert ours.get(k) == v, (k, ours.get(k), v)
    base = dict(ours)
    for r in ref["names"]:
        cfg = dict(base, case=r["case"], Mach=r["Mach"], aoa=r["aoa"])
        mesh = type("M", (), {"metadata": {} if r["h"] is None else {"h": r["h"]}})()
        assert Cfg.format_h(mesh) == r["h_tag"]
        assert Cfg.format_condition_tag(cfg) == r["condition"]
        assert Cfg.format_snapshot_name(cfg, r["t"]) == r["snapshot"]


def test_cli_configurations_match_reference():
    """euler/config.py:32-62: the configuration the command line builds, for
    the same argument lists, key by key (the package adds --precision)."""
    import json
    from eulersr_b200 import config as Cfg
    ref = json.loads((GOLDEN / "reference_config.json").read_text())
    for case in ref["cli"]:
        ours = Cfg.build_config_from_cli(Cfg.load_default_config(), case["argv"])
        for k, v in case["cfg"].items():
            assert ours.get(k) == v, (case["argv"], k, ours.get(k), v)


def test_run_summary_matches_reference(tmp_path):
    """euler/utils.py:147-191: the summary dictionary (keys, order, values)
    and the JSON file the reference writes for it, byte for byte."""
    import json
    from eulersr_b200 import main as M
    ref = json.loads((GOLDEN / "reference_summary.json").read_text())
    mesh = type("M", (), {"metadata": {"h": 0.025}, "tris": np.zeros((1234, 3), np.int32), "n_cells": 1234})()
    cfg = dict(case="naca0012", Mach=0.8, aoa=-2.5, time_scheme="SRK2", flux="HLLC", reconstruction="MUSCL",
               mesh_path="m.npy", stationarity_threshold=1e-5, stationarity_check_every=25)
    for r in ref:
        summ = M.build_run_summary(cfg, mesh, **r["kwargs"])
        assert summ == r["summary"]
        M.export_run_summary({"res": tmp_path}, summ, "AOA-2.50_M0.80_HLLC_MUSCL_SRK2_t1.00", verbose=False)
        assert (tmp_path / r["file"]).read_text() == r["text"]


def test_diamond_panels_match_reference_theory():
    """The shock-expansion states of the diamond's four faces (Mach, pressure
    ratio, Cp, shock angle, attached or detached) against the reference's own
    diamond_panels (euler/postproc/theory_validation_diamond.py:44-175)."""
    import json
    from eulersr_b200 import theory_validation as TV
    ref = json.loads((GOLDEN / "reference_theory.json").read_text())["panels"]
    for r in ref:
        ours = TV.diamond_panels(r["mach"], r["aoa"], 5.0)
        assert TV.all_attached(ours) == r["attached"], (r["mach"], r["aoa"])
        if not r["attached"]:
            continue
        for name, p in r["panels"].items():
            q = ours[name]
            assert q.regime == p["regime"], name
            assert q.M == pytest.approx(p["M"], rel=1e-8), (r["mach"], r["aoa"], name)
            assert q.p_ratio_freestream == pytest.approx(p["p_ratio"], rel=1e-8), name
            assert q.Cp == pytest.approx(p["Cp"], rel=1e-8, abs=1e-12), name
            if p["beta_deg"] is None:
                assert q.beta_deg is None, name
            else:
                assert q.beta_deg == pytest.approx(p["beta_deg"], abs=1e-6), name


def test_campaign_helpers_match_reference():
    """The validation campaigns' helpers against the reference's own on the
    same inputs: per-face plateau values of a wall profile, the leading-edge
    shock angle from a |grad p| field, the log-log order fit
    (theory_validation_diamond.py:237-342,609-621), the GCI triplets and the
    wall-profile error (mesh_convergence_diamond.py:106-161)."""
    import json
    from eulersr_b200 import mesh_convergence as MC
    from eulersr_b200 import theory_validation as TV
    h = json.loads((GOLDEN / "reference_theory.json").read_text())["helpers"]
    a = np.load(GOLDEN / "reference_theory_inputs.npz")
    prof = {k: a[f"profile_{k}"] for k in ("x", "y", "p", "mach")}
    masks = TV.panel_masks(prof, 1.5, 2.0)
    assert TV.plateau_value(prof, masks, "p", lambda p: (p - 1.0) / 2.8) == pytest.approx(h["plateau_p"], rel=1e-14)
    assert TV.plateau_value(prof, masks, "mach", lambda m: m) == pytest.approx(h["plateau_mach"], rel=1e-14)
    for side in ("upper", "lower"):
        got = TV.measure_shock_angle(a["shock_node_pos"], a["shock_grad_p"], 1.5, 2.0, 1.0, 0.0875, 0.0, side)
        assert got == pytest.approx(h["shock"][side], abs=1e-9), side
    p, r2, n = TV.fit_order(h["fit"]["rows"], "e")
    assert (p, r2, n) == (pytest.approx(h["fit"]["p"], rel=1e-12), pytest.approx(h["fit"]["r2"], rel=1e-12),
                          h["fit"]["n"])
    vals = {float(k): v for k, v in h["gci"]["values"].items()}
    ours = MC.richardson_gci(vals, h["gci"]["chain"])
    assert len(ours) == len(h["gci"]["triplets"])
    for o, r in zip(ours, h["gci"]["triplets"]):
        for k in ("h_coarse", "h_mid", "h_fine"):
            assert o[k] == r[k]
        for k in ("p_obs", "extrap", "gci_fine_pct"):
            assert o[k] == pytest.approx(r[k], rel=1e-12), k
    err = MC.relative_profile_error({"s": a["perr_ref_s"], "mach": a["perr_ref_mach"]},
                                    {"s": a["perr_cur_s"], "mach": a["perr_cur_mach"]})
    assert err == pytest.approx(h["profile_error"], rel=1e-12)



@pytest.mark.parametrize("tag,name,mach,aoa", [("diamond", "diamond_h0.2", 2.5, 5.0),
                                               ("naca", "naca0012_h0.2", 0.8, 1.25)])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_bitwise_equals_reference_solver_source(tag, name, mach, aoa, prec):
    """20 SRK2 steps of the oracle equal, bit for bit, those of EulerSR's own
    solver source (geometry, initialize, dt, boundary states, LSQ gradient,
    Venkatakrishnan limiter, MUSCL, HLLC, sponge, SSP-RK2) run with NumPy in
    place of jax.numpy (tests/golden/reference_solver_run.py), in float32 and
    float64, supersonic diamond and transonic NACA0012."""
    from conftest import oracle_mesh
    from oracle import euler_oracle as O
    ref = np.load(GOLDEN / "reference_solver.npz")
    dtype = np.float32 if prec == "f32" else np.float64
    mesh = load_mesh(name)
    om = oracle_mesh(mesh, dtype)
    W, inlet = O.initialize(mesh.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=mach, aoa=aoa,
                                               case=mesh.metadata["case"]), dtype)
    dt = O.get_dt(W, om, CFL=0.45 if 0.6 < mach < 1.1 else 0.6)
    assert dt == ref[f"{tag}_{prec}_dt"]
    for _ in range(20):
        W = O.time_step_srk2(W, om, dt, inlet)
    assert W.dtype == ref[f"{tag}_{prec}_W20"].dtype
    assert np.array_equal(W, ref[f"{tag}_{prec}_W20"])
    # the reference's CD, CL (helper.py:366-415) and entropy created (:312-320)
    W0, _ = O.initialize(mesh.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=mach, aoa=aoa,
                                            case=mesh.metadata["case"]), dtype)
    cd, cl = O.force_coefficients(W, om, 1.0, mach * 1.4 ** 0.5, mesh.metadata["obstacle_length"])
    ds = O.total_entropy(W, om) - O.total_entropy(W0, om)
    assert [cd, cl, float(ds)] == ref[f"{tag}_{prec}_cd_cl_dS"].tolist()


@pytest.mark.parametrize("flux,rec,scheme", [("Rusanov", "MUSCL", "SRK2"), ("HLLC", "constant", "SRK2"),
                                             ("HLLC", "MUSCL", "EE"), ("HLLC", "MUSCL", "RK2")])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_scheme_variants_equal_reference_source(flux, rec, scheme, prec):
    """The Rusanov flux, constant reconstruction, explicit Euler and RK2 of the
    oracle against the reference's own functions (euler_solver.py:201-244,
    106-122, 630-654), 10 steps of the diamond, bit for bit."""
    from conftest import oracle_mesh
    from oracle import euler_oracle as O
    ref = np.load(GOLDEN / "reference_solver.npz")
    dtype = np.float32 if prec == "f32" else np.float64
    mesh = load_mesh("diamond_h0.2")
    om = oracle_mesh(mesh, dtype)
    W, inlet = O.initialize(mesh.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.5, aoa=5.0,
                                               case="diamond"), dtype)
    dt = O.get_dt(W, om, CFL=0.6)
    fn = O.TIME_SCHEMES[scheme]
    for _ in range(10):
        W = fn(W, om, dt, inlet, reconstruction=rec.lower(), flux=flux.lower())
    assert np.array_equal(W, ref[f"variant_{flux}_{rec}_{scheme}_{prec}_W10"])


def test_freestream_equals_reference_initial_state():
    """The package's freestream state (what the solver fills a slot with) is
    the reference's initialize() state bit for bit, float32 and float64."""
    from eulersr_b200.solver import freestream
    ref = np.load(GOLDEN / "reference_solver.npz")
    from oracle import euler_oracle as O
    for dtype in (np.float32, np.float64):
        for mach, aoa in ((2.5, 5.0), (0.8, 1.25), (1.7, -3.3)):
            W, _ = O.initialize(3, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=mach, aoa=aoa, case="diamond"),
                                dtype)
            assert np.array_equal(freestream(mach, aoa, dtype=dtype), W[0])
    assert ref["diamond_f32_W20"].dtype == np.float32


@pytest.mark.parametrize("tag,name,prec", [("diamond", "diamond_h0.2", "f32"), ("diamond", "diamond_h0.2", "f64"),
                                           ("naca_eng", "naca0012_h0.2", "f32"),
                                           ("naca_eng", "naca0012_h0.2", "f64"),
                                           ("naca_cap", "naca0012_h0.2", "f64")])
def test_oracle_run_equals_reference_main_loop(tag, name, prec):
    """The oracle's run() against euler/main.py:43-270 itself (run with NumPy
    for jax.numpy, exports off): final state bit for bit, converged flag and
    stopping step of the stationarity rule, and the engineering criterion's
    confirmation and stopping step. Covers a stop at the first checks, a late
    stop with the engineering criterion confirmed early, and a case that
    reaches N unconverged."""
    import json
    from conftest import oracle_mesh
    from oracle import euler_oracle as O
    ref = np.load(GOLDEN / "reference_runs.npz")
    cfg = json.loads(str(ref["cfgs_json"]))[tag]
    dtype = np.float32 if prec == "f32" else np.float64
    mesh = load_mesh(name)
    om = oracle_mesh(mesh, dtype)
    W, inlet = O.initialize(mesh.n_cells, cfg, dtype)
    r = O.run(W, om, inlet, dict(cfg))
    conv, stop, eng_conv, eng_stop = (int(x) for x in ref[f"{tag}_{prec}_stop"])
    assert bool(r.converged) == bool(conv) and r.stopping_step == stop
    if "engineering_target_cd" in cfg:
        assert bool(r.eng_converged) == bool(eng_conv) and r.eng_stopping_step == eng_stop
    else:   # untracked: the reference reports None (euler/main.py:225-226)
        assert r.eng_converged is None and r.eng_stopping_step is None
    assert np.array_equal(r.W, ref[f"{tag}_{prec}_W"])


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_bitwise_equals_reference_solver_source_hr(prec):
    """The same pin at the HR size (h = 0.025): 20 SRK2 steps on the diamond
    h = 0.025 (19,384 cells, the package's mesher; the fixture records the
    mesh's digest), M 2.0, alpha 0, equal bit for bit to the reference's own
    source run with NumPy (tests/golden/reference_solver_hr.npz)."""
    from conftest import oracle_mesh
    from golden.make_reference_fixtures import mesh_digest
    from eulersr_b200.meshing.generate import cached_mesh
    from oracle import euler_oracle as O
    ref = np.load(GOLDEN / "reference_solver_hr.npz")
    mesh = cached_mesh("diamond", 0.025)
    assert str(ref["mesh_sha256"]) == mesh_digest(mesh)
    dtype = np.float32 if prec == "f32" else np.float64
    om = oracle_mesh(mesh, dtype)
    W, inlet = O.initialize(mesh.n_cells, dict(rho_inf=1.0, p_inf=1.0, gamma=1.4, Mach=2.0, aoa=0.0,
                                               case="diamond"), dtype)
    dt = O.get_dt(W, om, CFL=0.6)
    assert dt == ref[f"{prec}_dt"]
    for _ in range(20):
        W = O.time_step_srk2(W, om, dt, inlet)
    assert np.array_equal(W, ref[f"{prec}_W20"])
