"""The algorithmic byte counts behind the bench line's roofline and Dslash
figures, checked against their closed forms (no GPU needed)."""
import importlib.util
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", REPO / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("V,Ls", [(512 * 512, 16), (64 * 64, 16), (128 * 128, 24)])
def test_dslash_bytes_domain_wall(bench, V, Ls):
    # every spinor (2 spins) read and written once, two complex links per 4-D site
    assert bench.dslash_bytes(V, Ls, 8) == V * (64 * Ls + 32)
    assert bench.dslash_bytes(V, Ls, 4) == V * (32 * Ls + 16)


def test_dslash_bytes_wilson(bench):
    V = 2048 * 2048
    assert bench.dslash_bytes(V, 1, 8) == V * 96
    assert bench.dslash_bytes(V, 1, 4) == V * 48
    assert bench.WILSON_DSLASH_LATTICE == (2048, 2048)
    # both Dslash working sets (FP64 input and output fields) exceed the 126 MB L2
    assert 2 * V * 2 * 16 > 2 * 126e6
    Dt, Dx, Dl = bench.DSLASH_LATTICE
    assert 2 * Dt * Dx * Dl * 2 * 16 > 2 * 126e6


def test_even_odd_iteration_bytes(bench):
    V, Ls = 64 * 64, 16
    half_site = (V // 2) * Ls
    assert bench.eo_iter_bytes(V, Ls) == 17 * half_site * 16 + 8 * V * 8
    assert bench.eo_reliable_update_bytes(V, Ls) == 16 * half_site * 32 + 8 * V * 16


def test_cg_iteration_bytes(bench):
    V, Ls = 64 * 64, 16
    assert bench.cg_iter_bytes(V, Ls, 4) == 2 * bench.dslash_bytes(V, Ls, 4) + 10 * V * Ls * 16
    assert bench.reliable_update_bytes(V, Ls) == 2 * bench.dslash_bytes(V, Ls, 8) + V * Ls * 176
