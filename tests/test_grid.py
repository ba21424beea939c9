"""The grid driver's host logic (slurm/run_euler_grid.py:24-56,60-92) on CPU."""
from conftest import ROOT
from eulersr_b200 import grid as G


def test_parse_range():
    assert G.parse_range("0.7:1.0:0.1") == [0.7, 0.8, 0.9, 1.0]
    assert G.parse_range("-5:5:5") == [-5.0, 0.0, 5.0]
    assert G.parse_range("1,2.5, 3,") == [1.0, 2.5, 3.0]
    assert G.parse_range("2") == [2.0]
    # the step count rounds, so a range whose float steps drift keeps its end
    assert len(G.parse_range("0.7:3.0:0.01")) == 231


def test_normalize_optional_value():
    argv = ["--case", "diamond", "--aoa", "-5:5:1", "--mach", "2"]
    assert G.normalize_optional_value(argv, "--aoa") == ["--case", "diamond", "--aoa=-5:5:1", "--mach", "2"]
    assert G.normalize_optional_value(["--aoa", "--mach"], "--aoa") == ["--aoa", "--mach"]


def test_build_case_cfg():
    base = {"case": "diamond", "Mach": 1.0, "aoa": 2.0, "export": {"bundle": True}}
    c = G.build_case_cfg(base, "diamond", 1.23456789012345, -3.0)
    assert c["Mach"] == 1.2345678901 and c["aoa"] == -3.0 and c["stationarity_threshold"] == 1e-5
    assert G.build_case_cfg(base, "bump", 1.0, 4.0)["aoa"] == 0.0
    c["export"]["bundle"] = False
    assert base["export"]["bundle"] is True      # deep copy


def test_dry_run(capsys):
    rc = G.main(["--case", "diamond", "--mesh-path", str(ROOT / "tests" / "golden" / "diamond_h0.2.npz"),
                 "--mach", "1.5:2.0:0.5", "--aoa", "-2:2:2", "--dry-run"])
    out = capsys.readouterr().out
    assert rc == 0
    assert "Cases to run: 6" in out
    assert "case=diamond Mach=1.5 AoA=-2.0" in out and "case=diamond Mach=2.0 AoA=2.0" in out
