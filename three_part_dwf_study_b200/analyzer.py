"""The domain-wall analyzer over one or more GPUs: the reference's
analyze_domain_wall (domain_wall/analyze_configs.cpp:17-309) with its
per-configuration loop (:45-76) sharded across ranks.

Each rank takes a contiguous block of the configurations (shard.partition),
measures it in one batched call on its own GPU (DomainWall.measure: all point,
wall and Z4-noise propagators of the block in one persistent solve, then the
contractions), and the per-configuration outputs are all-gathered
(shard.gather_outputs; NCCL between GPUs). Rank 0 then runs the host
reductions (analysis.reduce_ensemble) and writes the reference's CSV files.
The Z4 noise of configuration c is drawn from mt19937_64(eta.random_seed +
104729 c) (analyze_configs.cpp:66-68) with c the global index, so the result
does not depend on the number of ranks.

    python -m three_part_dwf_study_b200.analyzer [--workdir DIR]
    torchrun --nproc-per-node N -m three_part_dwf_study_b200.analyzer [--workdir DIR]

reads DIR/parameters.txt and DIR/output/domain_wall/analysis_configs.npy and
writes DIR/output/domain_wall/{correlator,channels_by_config,
momentum_correlators}.csv.
"""
import argparse
import os
import sys
from pathlib import Path

import numpy as np

from . import _capi as A
from . import analysis, shard
from .params import TextConfig, dwf_parameters

CONFIGS = Path("output") / "domain_wall" / "analysis_configs.npy"
OUTDIR = Path("output") / "domain_wall"


def load_configs(path, Nt, Nx):
    """[n][2 Nt Nx] from the reference's analysis_configs.npy (shape (n, 2, Nt, Nx))."""
    a = np.load(path)
    if a.ndim != 4 or a.shape[1] != 2 or a.shape[2] != Nt or a.shape[3] != Nx:
        raise RuntimeError("analysis_configs.npy has the wrong shape")
    return np.ascontiguousarray(a, dtype=np.float64).reshape(a.shape[0], -1)


def measure_block(d, p, thetas, first, solver=A.SOLVER_EO_MIXED):
    """Per-configuration outputs of configurations first .. first + len(thetas) - 1."""
    from .rng import z4_digits
    n = thetas.shape[0]
    nn = p["eta_noise_vectors"]
    V = p["Nt"] * p["Nx"]
    z4 = None
    if nn > 0 and n > 0:
        z4 = np.concatenate([z4_digits(p["eta_random_seed"] + 104729 * (first + k), nn * V * 2)
                             for k in range(n)])
    if n == 0:
        return {"cpp": np.zeros((0, p["Nt"])), "cj5": np.zeros((0, p["Nt"])),
                "loop": np.zeros((0, V), np.complex128),
                "mom_cpp": np.zeros((0, p["max_momentum"] + 1, p["Nt"]))}
    m = d.measure(thetas, z4=z4, n_point_times=2, n_wall_times=2, n_noise=nn,
                  max_momentum=p["max_momentum"], rtol=p["propagator_rtol"],
                  maxiter=p["propagator_maxiter"], solver=solver)
    return {k: m[k] for k in ("cpp", "cj5", "loop", "mom_cpp")}


def analyze(workdir=".", world=1, rank=0, device=0, solver=A.SOLVER_EO_MIXED, comm_device=None,
            write=True):
    """Run the analyzer in `workdir` as rank `rank` of `world` (torch.distributed
    initialised by the caller when world > 1). Returns the ensemble reductions on
    every rank."""
    from .dwf import DomainWall
    wd = Path(workdir)
    p = dwf_parameters(TextConfig(wd / "parameters.txt"))
    thetas = load_configs(wd / CONFIGS, p["Nt"], p["Nx"])
    nconf = thetas.shape[0]
    first, _ = shard.partition(nconf, world, rank)
    d = DomainWall(p["Nt"], p["Nx"], p["N5"], p["M5"], p["mf"], p["beta"], device=device)
    try:
        meas = shard.sharded_measure(lambda th: measure_block(d, p, th, first, solver), thetas,
                                     world, rank, comm_device)
    finally:
        d.close()
    red = analysis.reduce_ensemble(meas, p["Nt"], p["Nx"], p["eta_flavors"])
    if write and rank == 0:
        analysis.write_csvs(red, meas["cpp"], wd / OUTDIR)
    return red


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workdir", default=".")
    ap.add_argument("--solver", type=int, default=A.SOLVER_EO_MIXED)
    a = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    comm_device = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        comm_device = torch.device("cuda", local)
    try:
        red = analyze(a.workdir, world, rank, local, a.solver, comm_device)
        if rank == 0:
            print(f"m_res = {red['m_res_average']:.6g} over {len(red['eta_all'])} configurations "
                  f"on {world} GPU(s)")
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
