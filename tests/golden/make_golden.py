#!/usr/bin/env python3
"""Regenerate the golden fixtures under tests/golden/ from the reference itself.

Runs in the build container only (it needs the reference sources): builds the
reference's own C++ (domain_wall/*.cpp, wilson/*.cpp and the driver programs in
oracle/ref_drivers, all compiled unmodified against the Eigen-API subset in
three_part_dwf_study_b200/host/eigen_shim) with ``make -C oracle ref REF=<checkout>``, then for each case writes a parameters.txt and seeded
inputs into a scratch directory, runs the reference there and copies the
outputs into tests/golden/<case>/.

Inputs are seeded synthetic fields: link phases uniform in [-pi, pi) and
complex Gaussian spinors, as the lattice study's hot starts and heatbaths use.

    python tests/golden/make_golden.py <reference checkout>
"""
import json
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF_BIN = REPO / "oracle" / "_ref"

BASE = {
    "wilson.Nt": 8, "wilson.Nx": 8, "wilson.beta": 2.0, "wilson.m0": 0.1,
    "wilson.trajectories": 4, "wilson.thermalization_cut": 1, "wilson.thin": 1,
    "wilson.hmc_steps": 5, "wilson.trajectory_length": 0.5,
    "wilson.source_t": 0, "wilson.source_x": 0,
    "wilson.time_boundary_sign": -1.0, "wilson.space_boundary_sign": 1.0,
    "wilson.force_cg_tolerance": 1.0e-12, "wilson.force_cg_max_iterations": 4000,
    "wilson.measurement_cg_tolerance": 1.0e-12,
    "wilson.measurement_cg_max_iterations": 4000, "wilson.random_seed": 1234,
    "dwf.Nt": 8, "dwf.Nx": 8, "dwf.N5": 4, "dwf.beta": 3.0, "dwf.M5": 1.0,
    "dwf.mf": 0.05, "dwf.epsilon": 0.05, "dwf.leapfrog_steps": 10,
    "dwf.trajectories": 4, "dwf.thermalization_cut": 1, "dwf.thin": 1,
    "dwf.pseudofermion_rtol": 1.0e-12, "dwf.pseudofermion_maxiter": 4000,
    "dwf.propagator_rtol": 1.0e-12, "dwf.propagator_maxiter": 4000,
    "dwf.random_seed": 1234,
    "eta.noise_vectors": 2, "eta.random_seed": 918273, "eta.flavors": 2,
    "analysis.threads": 1, "analysis.plateau_window_size": 2,
    "analysis.plateau_flatness_tolerance": 0.5, "analysis.earliest_plateau_time": 1,
    "analysis.fit_t_min": 1, "analysis.fit_t_max": 3, "analysis.gevp_t0": 1,
    "analysis.max_momentum": 3, "analysis.bootstrap_resamples": 10,
    "analysis.bootstrap_block_size": 1, "analysis.bootstrap_seed": 1,
}

# name -> (kind, overrides, input seed)
CASES = {
    "dwf_8x8x4": ("dwf", {}, 11),
    "dwf_6x10x3": ("dwf", {"dwf.Nt": 6, "dwf.Nx": 10, "dwf.N5": 3, "dwf.M5": 1.3,
                           "dwf.mf": 0.2, "analysis.max_momentum": 2}, 12),
    "dwf_hmc_8x8x4": ("dwf_hmc", {"dwf.mf": 0.2}, None),
    "wil_8x8": ("wil", {}, 21),
    "wil_6x10": ("wil", {"wilson.Nt": 6, "wilson.Nx": 10, "wilson.m0": 0.3,
                         "wilson.source_t": 2, "wilson.source_x": 3,
                         "wilson.space_boundary_sign": -1.0}, 22),
    "wil_hmc_8x8": ("wil_hmc", {"wilson.trajectories": 6, "wilson.m0": 0.3,
                                "wilson.trajectory_length": 0.5, "wilson.hmc_steps": 5,
                                "analysis.plateau_window_size": 2,
                                "analysis.plateau_flatness_tolerance": 10.0}, None),
}


def render(params):
    return "".join(f"{k} = {v!r}\n" if isinstance(v, float) else f"{k} = {v}\n"
                   for k, v in params.items())


def hot_theta(rng, nt, nx):
    return rng.uniform(-np.pi, np.pi, size=(2, nt, nx))


def gaussian_field(rng, n):
    return (rng.normal(size=(n, 2)) / np.sqrt(2.0))


def run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed:\n{r.stdout}\n{r.stderr}")
    return r.stdout


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    subprocess.run(["make", "-C", str(REPO / "oracle"), "ref", f"REF={sys.argv[1]}"], check=True)
    for name, (kind, over, seed) in CASES.items():
        params = dict(BASE)
        params.update(over)
        dest = HERE / name
        if dest.exists():
            shutil.rmtree(dest)
        dest.mkdir(parents=True)
        with tempfile.TemporaryDirectory() as tmp:
            tmp = Path(tmp)
            (tmp / "parameters.txt").write_text(render(params))
            if kind == "dwf":
                nt, nx, ls = params["dwf.Nt"], params["dwf.Nx"], params["dwf.N5"]
                rng = np.random.default_rng(seed)
                np.save(tmp / "in_theta.npy", hot_theta(rng, nt, nx))
                np.save(tmp / "in_psi.npy", gaussian_field(rng, ls * nt * nx * 2))
                np.save(tmp / "in_chi.npy", gaussian_field(rng, ls * nt * nx * 2))
                run([str(REF_BIN / "dwf_golden")], tmp)
            elif kind == "wil":
                nt, nx = params["wilson.Nt"], params["wilson.Nx"]
                rng = np.random.default_rng(seed)
                np.save(tmp / "in_theta.npy", hot_theta(rng, nt, nx))
                np.save(tmp / "in_psi.npy", gaussian_field(rng, nt * nx * 2))
                run([str(REF_BIN / "wilson_golden")], tmp)
            elif kind == "dwf_hmc":
                (tmp / "output" / "domain_wall").mkdir(parents=True)
                run([str(REF_BIN / "generate_domain_wall")], tmp)
                run([str(REF_BIN / "analyze_domain_wall")], tmp)
                for f in ["configs.npy", "analysis_configs.npy", "run_info_history.csv",
                          "correlator.csv", "channels_by_config.csv",
                          "momentum_correlators.csv"]:
                    shutil.copy2(tmp / "output" / "domain_wall" / f, dest / f)
            elif kind == "wil_hmc":
                (tmp / "output" / "wilson").mkdir(parents=True)
                run([str(REF_BIN / "generate_wilson")], tmp)
                run([str(REF_BIN / "analyze_wilson")], tmp)
                for f in ["wilson_ensemble.bin", "hmc_history.csv",
                          "correlators_by_config.csv"]:
                    shutil.copy2(tmp / "output" / "wilson" / f, dest / f)
            for f in sorted(tmp.glob("*.npy")):
                shutil.copy2(f, dest / f.name)
            shutil.copy2(tmp / "parameters.txt", dest / "parameters.txt")
        (dest / "case.json").write_text(json.dumps({"kind": kind, "params": params}, indent=1))
        print("wrote", dest.relative_to(REPO))


if __name__ == "__main__":
    sys.exit(main())
