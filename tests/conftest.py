import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the native library")
    # temporary files of the tests stay inside the checkout
    if not config.option.basetemp:
        config.option.basetemp = str(ROOT / ".pytest_tmp")


@pytest.fixture(scope="session")
def golden():
    return GOLDEN


def load_mesh(name):
    from eulersr_b200.mesh import Mesh
    return Mesh.load(GOLDEN / f"{name}.npz")


@pytest.fixture(scope="session")
def diamond02():
    return load_mesh("diamond_h0.2")


@pytest.fixture(scope="session")
def naca02():
    return load_mesh("naca0012_h0.2")


@pytest.fixture(scope="session")
def diamond01():
    return load_mesh("diamond_h0.1")


def oracle_mesh(mesh, dtype):
    from oracle import euler_oracle as O
    return O.build_oracle_mesh(mesh.points, mesh.tris, mesh.neighbors, mesh.faces, mesh.face_markers,
                               mesh.face_connectivity, dtype=dtype, metadata=mesh.metadata)


def rel_err(a, b):
    """max |a-b| per field over max |b| per field (field-scaled relative error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b).max(0) / np.maximum(np.abs(b).max(0), 1e-300)))
