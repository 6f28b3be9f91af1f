"""The reference's own four mains, compiled unmodified against the drop-in
headers (three_part_dwf_study_b200/host/dropin) so that every hot-path call
runs on the GPU through libdwfb200.so, reproduce the reference's own runs
(tests/golden/dwf_hmc_8x8x4, wil_hmc_8x8): same accept decisions and
configurations (1e-9 relative), same CSV outputs (6 significant digits, 2e-5).
Three solver settings are exercised: DWF_B200_SOLVER=cg64 (the reference's
FP64 CG everywhere), =mixed (the full-lattice mixed FP32/FP64 CG everywhere)
and the default (mixed CG in HMC, even-odd Schur mixed CG for the analyzers'
propagators)."""
import csv
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import REPO, rel

pytestmark = pytest.mark.gpu

BIN = REPO / "three_part_dwf_study_b200" / "host" / "_bin"


def run(name, cwd, solver):
    exe = BIN / name
    if not exe.exists():
        pytest.skip(f"{exe} not built (needs the reference sources at build time)")
    # DWF_B200_DEVICE=auto: the device is handed out in turn (one GPU here: 0)
    env = dict(os.environ, DWF_B200_SOLVER=solver, DWF_B200_DEVICE="auto", TMPDIR=str(cwd))
    r = subprocess.run([str(exe)], cwd=cwd, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def table(path):
    rows = list(csv.DictReader(open(path)))
    return np.array([[float(v) for v in r.values()] for r in rows])


@pytest.mark.parametrize("solver", ["cg64", "mixed", "default"])
def test_dropin_domain_wall_generate_and_analyze(golden, tmp_path, solver):
    g = golden("dwf_hmc_8x8x4")
    shutil.copy2(g.dir / "parameters.txt", tmp_path / "parameters.txt")
    (tmp_path / "output" / "domain_wall").mkdir(parents=True)
    run("generate_domain_wall", tmp_path, solver)
    out = tmp_path / "output" / "domain_wall"
    ours, ref = np.load(out / "configs.npy"), g.npy("configs.npy")
    assert ours.shape == ref.shape and rel(ours, ref) < 1e-9
    assert rel(np.load(out / "analysis_configs.npy"), g.npy("analysis_configs.npy")) < 1e-9
    h, hr = table(out / "run_info_history.csv"), table(g.dir / "run_info_history.csv")
    assert np.array_equal(h[:, 1], hr[:, 1])  # accepted
    assert np.allclose(h, hr, rtol=2e-5, atol=1e-9)
    run("analyze_domain_wall", tmp_path, solver)
    for name in ["correlator.csv", "channels_by_config.csv", "momentum_correlators.csv"]:
        a, b = table(out / name), table(g.dir / name)
        assert a.shape == b.shape, name
        assert np.allclose(a, b, rtol=2e-5, atol=1e-12 * np.abs(b).max()), name


@pytest.mark.parametrize("solver", ["cg64", "mixed", "default"])
def test_dropin_wilson_generate_and_analyze(golden, tmp_path, solver):
    g = golden("wil_hmc_8x8")
    shutil.copy2(g.dir / "parameters.txt", tmp_path / "parameters.txt")
    (tmp_path / "output" / "wilson").mkdir(parents=True)
    run("generate_wilson", tmp_path, solver)
    out = tmp_path / "output" / "wilson"
    ours, ref = (out / "wilson_ensemble.bin").read_bytes(), (g.dir / "wilson_ensemble.bin").read_bytes()
    assert len(ours) == len(ref) and ours[:40] == ref[:40]  # WILCFG1 header
    a = np.frombuffer(ours[40:], dtype=np.float64)
    b = np.frombuffer(ref[40:], dtype=np.float64)
    assert rel(a, b) < 1e-9
    h, hr = table(out / "hmc_history.csv"), table(g.dir / "hmc_history.csv")
    assert np.array_equal(h[:, 1], hr[:, 1])
    assert np.allclose(h, hr, rtol=2e-5, atol=1e-9)
    run("analyze_wilson", tmp_path, solver)
    a, b = table(out / "correlators_by_config.csv"), table(g.dir / "correlators_by_config.csv")
    assert a.shape == b.shape and np.allclose(a, b, rtol=2e-5)


@pytest.mark.parametrize("solver", ["cg64", "mixed"])
def test_dropin_conjugate_gradient_forms(golden, tmp_path, solver):
    """The drop-in conjugate_gradient in both forms (tests/dropin_src/cg_forms.cpp):
    the named normal operator, the reference's std::function signature
    (domain_wall/include/cg_solver.hpp:17-22) holding a b200::NormalOperator
    (the same GPU solve: identical iterations and solution) and holding the
    caller's own lambda over apply_D_dagger_D (host recurrences around the GPU
    operator: same solution to CG accuracy)."""
    g = golden("dwf_8x8x4")
    shutil.copy2(g.dir / "parameters.txt", tmp_path / "parameters.txt")
    out = run("cg_forms", tmp_path, solver)
    rows = {ln.split()[0]: ln.split()[1:] for ln in out.strip().splitlines()}
    assert set(rows) == {"named", "normal_operator", "lambda"}
    for name, (it, conv, rr, dx) in rows.items():
        assert int(conv) == 1 and float(rr) <= 1e-12, name
    assert rows["normal_operator"][0] == rows["named"][0]
    assert float(rows["normal_operator"][3]) == 0.0
    assert abs(int(rows["lambda"][0]) - int(rows["named"][0])) <= 3 or solver != "cg64"
    assert float(rows["lambda"][3]) < 1e-9
