import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def cfield(a):
    """(n, 2) float64 -> complex128."""
    return a[:, 0] + 1j * a[:, 1]


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


class Golden:
    def __init__(self, name):
        self.dir = GOLDEN / name
        self.case = json.loads((self.dir / "case.json").read_text())
        self.p = self.case["params"]

    def npy(self, name):
        return np.load(self.dir / name)

    def field(self, name):
        return cfield(self.npy(name))


@pytest.fixture(scope="session")
def golden():
    return Golden


def random_theta(rng, nt, nx):
    return rng.uniform(-np.pi, np.pi, size=2 * nt * nx)


def random_field(rng, n):
    return (rng.normal(size=n) + 1j * rng.normal(size=n)) / np.sqrt(2.0)


def quenched_theta(rng, nt, nx, beta):
    """Seeded pure-gauge configuration (see three_part_dwf_study_b200.ensemble)."""
    from three_part_dwf_study_b200.ensemble import quenched_theta as q
    return q(rng, nt, nx, beta)
