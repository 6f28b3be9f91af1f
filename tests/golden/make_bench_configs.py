#!/usr/bin/env python3
"""Generate the benchmark's gauge configurations with the GPU HMC.

DWF 64x64, Ls = 16, M5 = 1.0, m_f = 0.05, beta = 3.0: one Markov chain of the
reference generator's loop (three_part_dwf_study_b200.ensemble.hmc_chain: the
reference's draws, leapfrog epsilon = 0.01 with 40 steps, Metropolis) started
from a seeded pure-gauge configuration, pseudofermion solves by the mixed
FP32/FP64 CG to 1e-10; 10 thermalisation trajectories, then every second
configuration is kept until 12 are saved: configurations 0-7 are the per-rank
propagator workloads, 8-11 the learned preconditioner's training set. Written
to tests/golden/bench_hmc_64x64x16/configs.npy ([12][2*64*64] float64, the
reference's gauge_index layout) with a description beside it. Needs a GPU:

    python tests/golden/make_bench_configs.py
"""
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

NT, NX, LS, M5, MF, BETA = 64, 64, 16, 1.0, 0.05, 3.0
SEED, START_SEED = 20260101, 20260101
EPS, STEPS, THERM, THIN, KEEP = 0.01, 40, 10, 2, 12
OUT = HERE / "bench_hmc_64x64x16"


def main():
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200.ensemble import hmc_chain, quenched_theta
    d = T.DomainWall(NT, NX, LS, M5, MF, BETA)
    th0 = quenched_theta(np.random.default_rng(START_SEED), NT, NX, BETA)
    ntraj = THERM + THIN * (KEEP - 1) + 1
    t0 = time.time()
    cfg, hist = hmc_chain(d, th0, ntraj, seed=SEED, epsilon=EPS, steps=STEPS, rtol=1e-10,
                          maxiter=20000, solver=T.SOLVER_MIXED, thermalization_cut=THERM, thin=THIN)
    d.close()
    assert cfg.shape[0] == KEEP, cfg.shape
    OUT.mkdir(exist_ok=True)
    np.save(OUT / "configs.npy", cfg)
    (OUT / "case.json").write_text(json.dumps({
        "lattice": [NT, NX, LS], "M5": M5, "mf": MF, "beta": BETA,
        "start": f"ensemble.quenched_theta(default_rng({START_SEED}))",
        "chain": {"seed": SEED, "epsilon": EPS, "leapfrog_steps": STEPS, "trajectories": ntraj,
                  "thermalization_cut": THERM, "thin": THIN, "solver": "mixed CG to 1e-10"},
        "acceptance": float(hist["accepted"].mean()),
        "plaquette_kept": [float(v) for v in hist["plaquette"][THERM::THIN]],
        "use": "configs 0-7: per-rank propagator workload; 8-11: learned-preconditioner training",
        "seconds": round(time.time() - t0, 1)}, indent=1) + "\n")
    print(f"wrote {OUT / 'configs.npy'}: acceptance {hist['accepted'].mean():.2f}, "
          f"plaquette {hist['plaquette'][-1]:.4f}")


if __name__ == "__main__":
    main()
