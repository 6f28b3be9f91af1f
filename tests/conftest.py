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
    """Seeded 2-D U(1) gauge field with plaquette angles drawn independently
    from exp(beta cos P) (built in an axial gauge, then gauge-randomised);
    the periodic closure leaves one plaquette per slice off that law."""
    P = rng.vonmises(0.0, beta, size=(nt, nx))
    th = np.zeros((2, nt, nx))
    th[1, 0] = rng.uniform(-np.pi, np.pi, nx)
    for t in range(nt - 1):
        th[1, t + 1] = th[1, t] + P[t]
    for x in range(nx - 1):
        th[0, nt - 1, x + 1] = th[0, nt - 1, x] + th[1, 0, x] - th[1, nt - 1, x] - P[nt - 1, x]
    phi = rng.uniform(-np.pi, np.pi, (nt, nx))
    th[0] += phi - np.roll(phi, -1, 0)
    th[1] += phi - np.roll(phi, -1, 1)
    return np.angle(np.exp(1j * th)).ravel()
