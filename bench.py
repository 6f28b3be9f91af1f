#!/usr/bin/env python3
"""Benchmark: domain-wall propagator solves per second to a true FP64
residual of 1e-10 on one B200, and the standalone Dslash bandwidth (domain
wall at 512x512x16 and Wilson at 2048x2048, the autotuned kernels, which the
line names in `kernel_variant`).

Workload (one "step"): the per-configuration propagator set of the
domain-wall analyzer on a 64x64 lattice, Ls = 16, M5 = 1.0, m_f = 0.05 on a
beta = 3.0 gauge configuration thermalised by the GPU HMC (one chain of the
reference generator's loop, tests/golden/make_bench_configs.py): 2 spins x 4 source
times boundary point sources, 16 complex Z4 boundary-noise sources and
2 spins x 2 source times boundary wall sources (28 right-hand sides), each
solved as x = (D^dag D)^-1 D^dag src (domain_wall/include/correlator.hpp
:60-79, :129-142, :197-220) until the FP64 true residual of the normal
equation is <= 1e-10.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0. `value` = right-hand sides solved per second across
all ranks by the fastest of the solvers measured (even-odd mixed CG, or the
learned-preconditioned flexible GCR, whose network is trained on four
other configurations of the same HMC chain; training time reported apart),
inputs resident in HBM, CUDA-event device time, max over ranks;
`e2e` = the same through the host C-ABI entry (dwf_set_gauge + dwf_propagators
from pinned host buffers, solutions read back). With --gpus N (torchrun) every
rank solves its own configuration's set (weak scaling, no exchange).
`--impl reference` times the reference's own CPU solver (oracle/_ref/ref_bench,
the reference's conjugate_gradient + apply_D_dagger_D compiled from its
sources) on the host cores instead.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

NT, NX, LS = 64, 64, 16
M5, MF, BETA = 1.0, 0.05, 3.0
RTOL = 1.0e-10
MAXITER = 20000
N_NOISE = 16
GAUGE_SEED = 20260101
NOISE_SEED = 918273
REF_BENCH = REPO / "oracle" / "_ref" / "ref_bench"
DSLASH_LATTICE = (512, 512, 16)
L2_FLUSH_BYTES = 256 << 20


BENCH_CONFIGS = REPO / "tests" / "golden" / "bench_hmc_64x64x16" / "configs.npy"


def bench_configs():
    """Configurations of one GPU-HMC Markov chain at the workload's parameters
    (tests/golden/make_bench_configs.py): 0-7 per-rank workloads, 8-11 the
    learned preconditioner's training set."""
    if not BENCH_CONFIGS.exists():
        raise SystemExit(f"{BENCH_CONFIGS} is missing: run tests/golden/make_bench_configs.py on a GPU")
    return np.load(BENCH_CONFIGS)


def workload_gauge(rank):
    return bench_configs()[rank % 8].copy()


def training_gauges(rank):
    return bench_configs()[8:12].copy()


LP_HIDDEN = 32
LP_TRAIN = dict(steps=4000, batch=8, lr=3e-3, lr_decay_steps=1333, pairs_per_conf=32,
                solver_iters=50, solver_every=2, solver_maxiter=20000, seed=11)


def boundary_source_set(Nt, Nx, Ls, seed):
    """28 boundary sources (complex128 [28, Ndof]): 2 spins at 4 point-source
    times (0, Nt/4, Nt/2, 3Nt/4), 16 Z4 noise vectors, 2 spins at 2 wall times
    (0, Nt/2). P_L = diag(0, 1), P_R = diag(1, 0): spin 1 of the source sits on
    s = 0, spin 0 on s = Ls-1 (correlator.hpp:133-138, :201-211, :60-75)."""
    srcs = []
    for t in (0, Nt // 4, Nt // 2, 3 * Nt // 4):
        for b in (0, 1):
            v = np.zeros((Ls, Nt, Nx, 2), np.complex128)
            if b == 1:
                v[0, t, 0, 1] = 1.0
            else:
                v[Ls - 1, t, 0, 0] = 1.0
            srcs.append(v.ravel())
    rng = np.random.default_rng(seed)
    phases = np.array([1, 1j, -1, -1j])
    for _ in range(N_NOISE):
        eta = phases[rng.integers(0, 4, size=(Nt, Nx, 2))]
        v = np.zeros((Ls, Nt, Nx, 2), np.complex128)
        v[0, :, :, 1] = eta[:, :, 1]
        v[Ls - 1, :, :, 0] += eta[:, :, 0]
        srcs.append(v.ravel())
    for t in (0, Nt // 2):
        for b in (0, 1):
            v = np.zeros((Ls, Nt, Nx, 2), np.complex128)
            if b == 1:
                v[0, t, :, 1] = 1.0
            else:
                v[Ls - 1, t, :, 0] = 1.0
            srcs.append(v.ravel())
    return np.stack(srcs)


def workload_sources(rank):
    """The workload's 28 boundary sources (boundary_source_set on the bench
    lattice; the noise seeded per rank)."""
    return boundary_source_set(NT, NX, LS, NOISE_SEED + 104729 * rank)


def sig(x, n=4):
    """x rounded to n significant digits (keeps the printed line short)."""
    if x is None or not np.isfinite(x) or x == 0:
        return x
    return float(f"{x:.{n}g}")


def measured_tensor_peak():
    """Measured dense BF16 TFLOP/s (burst) of this pool, else the fallback."""
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            v = json.loads(p.read_text()).get("bf16_tflops")
            if v:
                return float(v)
        except (ValueError, OSError):
            pass
    return 1590.0


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# algorithmic bytes (per right-hand side)
# ---------------------------------------------------------------------------
def dslash_bytes(V, Ls, w):
    """One D or D^dag application: every spinor read once and written once,
    links (complex) shared by the Ls slices: V * (Ls * 2 * 4w + 2 * 2w)."""
    return V * (Ls * 2 * 4 * w + 2 * 2 * w)


def cg_iter_bytes(V, Ls, w):
    """One CG iteration on D^dag D: two Dslash plus ten spinor streams."""
    return 2 * dslash_bytes(V, Ls, w) + 10 * V * Ls * 4 * w


def reliable_update_bytes(V, Ls):
    """FP64 residual replacement: two FP64 Dslash plus x, e, b reads and
    x, r, r32, e writes."""
    return 2 * dslash_bytes(V, Ls, 8) + V * Ls * (32 + 16 + 32 + 32 + 32 + 16 + 16)


def eo_iter_bytes(V, Ls):
    """One FP32 iteration of the even-odd Schur CG: 17 half-lattice spinor
    streams of 16 B per site (P1 2, P2 3, P3 2, P4 7, P5 3) and the FP32 links
    (2V x 8 B) once in each of the four operator phases."""
    return 17 * (V // 2) * Ls * 16 + 4 * 2 * V * 8


def eo_reliable_update_bytes(V, Ls):
    """FP64 residual replacement of the Schur normal equation: 16 half-lattice
    FP64-equivalent streams (x, e, y, t, b, parked x+e, r, r32, e32) and the
    FP64 links in four operator phases."""
    return 16 * (V // 2) * Ls * 32 + 4 * 2 * V * 16


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        smax = max(r[1] for r in rows)
        loaded = [r for r in rows if r[0] > 0.5 * smax] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in loaded for i, v in enumerate(r[2]) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU reference (the reference's own solver, compiled from its sources)
# ---------------------------------------------------------------------------
def ref_params_text(maxiter, Nt=NT, Nx=NX, Ls=LS):
    keys = {
        "wilson.Nt": 8, "wilson.Nx": 8, "wilson.beta": 2.0, "wilson.m0": 0.1,
        "wilson.trajectories": 1, "wilson.thermalization_cut": 0, "wilson.thin": 1,
        "wilson.hmc_steps": 1, "wilson.trajectory_length": 1.0, "wilson.source_t": 0,
        "wilson.source_x": 0, "wilson.time_boundary_sign": -1.0,
        "wilson.space_boundary_sign": 1.0, "wilson.force_cg_tolerance": 1e-10,
        "wilson.force_cg_max_iterations": 1, "wilson.measurement_cg_tolerance": 1e-10,
        "wilson.measurement_cg_max_iterations": 1, "wilson.random_seed": 1,
        "dwf.Nt": Nt, "dwf.Nx": Nx, "dwf.N5": Ls, "dwf.beta": BETA, "dwf.M5": M5,
        "dwf.mf": MF, "dwf.epsilon": 0.01, "dwf.leapfrog_steps": 1, "dwf.trajectories": 1,
        "dwf.thermalization_cut": 0, "dwf.thin": 1, "dwf.pseudofermion_rtol": RTOL,
        "dwf.pseudofermion_maxiter": maxiter, "dwf.propagator_rtol": RTOL,
        "dwf.propagator_maxiter": maxiter, "dwf.random_seed": 1, "eta.noise_vectors": 1,
        "eta.random_seed": 1, "eta.flavors": 2, "analysis.threads": 0,
        "analysis.plateau_window_size": 2, "analysis.plateau_flatness_tolerance": 0.1,
        "analysis.earliest_plateau_time": 1, "analysis.fit_t_min": 1, "analysis.fit_t_max": 2,
        "analysis.gevp_t0": 1, "analysis.max_momentum": 1, "analysis.bootstrap_resamples": 1,
        "analysis.bootstrap_block_size": 1, "analysis.bootstrap_seed": 1,
    }
    return "".join(f"{k} = {v!r}\n" if isinstance(v, float) else f"{k} = {v}\n"
                   for k, v in keys.items())


class RefWorkdir:
    """Scratch directory for the reference's timing driver (oracle/_ref/ref_bench):
    parameters.txt, the workload configuration and its 28 sources."""

    def __init__(self, rank=0, lattice=None, theta=None, sources=None):
        self.rank, self.lattice, self.theta, self.sources = rank, lattice, theta, sources

    def __enter__(self):
        self.tmp = tempfile.TemporaryDirectory()
        d = Path(self.tmp.name)
        Nt, Nx, Ls = self.lattice or (NT, NX, LS)
        (d / "parameters.txt").write_text(ref_params_text(MAXITER, Nt, Nx, Ls))
        th = workload_gauge(self.rank) if self.theta is None else self.theta
        np.save(d / "in_theta.npy", np.asarray(th, np.float64).reshape(2, Nt, Nx))
        src = workload_sources(self.rank) if self.sources is None else self.sources
        np.save(d / "in_src.npy", np.ascontiguousarray(src).view(np.float64).reshape(
            src.shape[0], -1, 2))
        self.dir = d
        return self

    def __exit__(self, *a):
        self.tmp.cleanup()

    def run(self, *args):
        r = subprocess.run([str(REF_BENCH)] + [str(a) for a in args], cwd=self.dir,
                           capture_output=True, text=True, timeout=3600)
        if r.returncode != 0:
            raise RuntimeError(f"ref_bench {args} failed: {r.stderr.strip()}")
        return json.loads(r.stdout.strip().splitlines()[-1])


def ref_solve_batch(wd, first, threads, nsrc=28):
    """One complete batch: min(threads, nsrc) concurrent complete solves (one
    per host thread) of the workload's sources first, first+1, ... (cycling
    through the 28); returns (solves, seconds, result)."""
    n = min(threads, nsrc)
    res = wd.run("solve", n, first % nsrc, n)
    if not all(res["converged"]):
        raise SystemExit(f"reference solves did not converge: {res}")
    return n, res["seconds"], res


def cpu_sample(threads, rank=0):
    """The CPU baseline beside the GPU line: one complete batch of the
    reference's solves (all host threads, one solve each). Returns
    (solves/s, description)."""
    if not REF_BENCH.exists():
        return None
    with RefWorkdir(rank) as wd:
        n, secs, res = ref_solve_batch(wd, 0, threads)
    desc = (f"one complete batch: {n} concurrent complete solves (one per host thread) of the "
            f"workload's first {n} sources (point, then Z4 noise), the reference's "
            f"apply_D_dagger + conjugate_gradient(apply_D_dagger_D) to rtol {RTOL:g}, "
            f"{min(res['iterations'])}-{max(res['iterations'])} iterations, {secs:.1f} s")
    return n / secs, desc


def cpu_apply_gbs(lattice, reps):
    """B1: the reference's apply_D on one host thread (its operator is serial),
    as equivalent GB/s with the same algorithmic bytes as the GPU Dslash."""
    Nt, Nx, Ls = lattice
    th = np.random.default_rng(3).uniform(-np.pi, np.pi, 2 * Nt * Nx)
    src = np.zeros((1, Ls * Nt * Nx * 2), np.complex128)
    with RefWorkdir(lattice=lattice, theta=th, sources=src) as wd:
        res = wd.run("apply", reps)
    t = res["seconds"] / reps
    return {"lattice": list(lattice), "ms_per_apply": round(t * 1e3, 2),
            "GBs": round(dslash_bytes(Nt * Nx, Ls, 8) / t / 1e9, 2), "threads": 1}


# ---------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def impl_reference(args):
    """The reference arm: the reference's own CPU solver on all host threads,
    complete solves of the workload's 28 sources. A step is one complete batch
    (one solve per thread, sources taken in turn through the 28), so every
    step is whole solves at rtol 1e-10 and `ms_per_step` is its wall time.
    Warm-up steps are one operator application each (page-in; a CPU needs no
    other warm-up)."""
    ws, rank, local = dist_setup()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    if not REF_BENCH.exists():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/ref_bench is not built"}))
        return 0
    secs, solves, iters = [], 0, []
    n = min(threads, 28)
    with RefWorkdir(rank) as wd:
        for _ in range(args.warmup):
            wd.run("apply", 1)
        for k in range(args.steps):
            m, t, res = ref_solve_batch(wd, k * n, threads)
            secs.append(t)
            solves += m
            iters += res["iterations"]
    value = solves / sum(secs)
    line = {
        "impl": "reference", "metric": "dwf_propagator_solves_per_s_true_res_1e-10",
        "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(secs) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config("reference CPU CG (FP64)"),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads,
                         "kind": "reference",
                         "sample": (f"each step {n} concurrent complete solves (one per host "
                                    f"thread) of the workload's 28 sources in turn, "
                                    f"{min(iters)}-{max(iters)} CG iterations each; warm-up "
                                    f"steps one apply_D each")},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


HMC_EPS, HMC_STEPS = 0.01, 40  # the reference's dwf.epsilon and dwf.leapfrog_steps


def hmc_compare(T, d, rank, ntraj, theta=None, lattice=None, seed=1234, maxiter=MAXITER):
    """ntraj domain-wall HMC trajectories from `theta` (default: the workload
    configuration), each run twice from identical momenta and pseudofermion
    draws (libstdc++ streams, the reference's order: chi then pi):
    pseudofermion solves by the plain FP64 CG and by the mixed CG, both to
    1e-10. Reports device time per trajectory (CUDA events on the library
    stream around the whole trajectory), dH of each and their largest
    difference, and the plaquette."""
    import torch
    from three_part_dwf_study_b200.rng import Rng
    if ntraj < 1:
        return None
    stream = torch.cuda.ExternalStream(d.stream_ptr())
    if theta is None:
        theta = workload_gauge(rank)
    rng = Rng(seed + rank)
    res = {"lattice": list(lattice or (NT, NX, LS)), "epsilon": HMC_EPS,
           "leapfrog_steps": HMC_STEPS, "rtol": RTOL, "trajectories": ntraj}
    per = {T.SOLVER_CG64: [], T.SOLVER_MIXED: []}
    dh = {T.SOLVER_CG64: [], T.SOLVER_MIXED: []}
    plaq = []
    for k in range(ntraj):
        chi = rng.pseudofermion(d.Ndof)
        mom = rng.normals(d.Ngauge)
        outs = {}
        for solver in (T.SOLVER_CG64, T.SOLVER_MIXED):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            out, info = d.hmc_trajectory(theta, chi, mom, HMC_EPS, HMC_STEPS, rtol=RTOL,
                                         maxiter=maxiter, solver=solver)
            e1.record(stream)
            e1.synchronize()
            per[solver].append(e0.elapsed_time(e1) * 1e-3)
            dh[solver].append(info["dH"])
            outs[solver] = (out, info)
        out, info = outs[T.SOLVER_CG64]
        plaq.append(info["plaquette"])
        if np.random.default_rng(k).uniform() < min(1.0, float(np.exp(-info["dH"]))):
            theta = out
    for solver, name in ((T.SOLVER_CG64, "plain_fp64_cg"), (T.SOLVER_MIXED, "mixed_cg")):
        res[name] = {"seconds_per_trajectory": statistics.mean(per[solver]), "dH": dh[solver]}
    res["max_abs_dH_difference"] = max(abs(a - b) for a, b in zip(dh[T.SOLVER_CG64], dh[T.SOLVER_MIXED]))
    res["speedup_mixed_vs_fp64"] = res["plain_fp64_cg"]["seconds_per_trajectory"] / \
        res["mixed_cg"]["seconds_per_trajectory"]
    res["plaquette"] = plaq
    return res


def analysis_batches(T, local, nconf=8):
    """The batched analyzer on the finite-volume scan's extremes (Nt = 64,
    Nx = 32 and 96, Ls = 16, m_f = 0.05, seeded beta = 3 configurations):
    nconf configurations per call, each with 2 spins x 4 point-source times,
    16 boundary Z4 noise sources and 2 spins x 2 wall-source times (28
    right-hand sides), solved together by the even-odd mixed solver to 1e-10
    and contracted (C_PP, C_J5, loop, momentum C_PP). Device time of the call
    (CUDA events on the library stream, host copies of configurations and
    correlators included) per configuration and per right-hand side."""
    import torch
    from three_part_dwf_study_b200.ensemble import quenched_theta
    from three_part_dwf_study_b200.rng import z4_digits
    out = {}
    for Nx in (32, 96):
        Nt, Ls = 64, 16
        d = T.DomainWall(Nt, Nx, Ls, M5, MF, BETA, device=local)
        st = torch.cuda.ExternalStream(d.stream_ptr())
        rng = np.random.default_rng(GAUGE_SEED + Nx)
        th = np.stack([quenched_theta(rng, Nt, Nx, BETA) for _ in range(nconf)])
        z4 = np.concatenate([z4_digits(NOISE_SEED + 104729 * k, N_NOISE * Nt * Nx * 2)
                             for k in range(nconf)])
        kw = dict(z4=z4, n_point_times=4, n_wall_times=2, n_noise=N_NOISE, max_momentum=5,
                  rtol=RTOL, maxiter=MAXITER, solver=T.SOLVER_EO_MIXED)
        d.measure(th, **kw)  # warm-up (autotuning, allocations)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        m = d.measure(th, **kw)
        e1.record(st)
        e1.synchronize()
        sec = e0.elapsed_time(e1) * 1e-3
        if not all(i["converged"] for i in m["info"]):
            raise SystemExit(f"analysis batch did not converge (Nx={Nx})")
        nr = len(m["info"])
        out[f"64x{Nx}x16"] = {"configurations": nconf, "rhs": nr,
                              "seconds_per_configuration": sec / nconf,
                              "solves_per_s": nr / sec,
                              "schur_iterations_mean": statistics.mean(i["schur_iterations"] for i in m["info"])}
        d.close()
    return out


def analysis_study(nconf=64, therm=10):
    """The finite-volume scan's analysis at full size: for each Nx in {32, 56,
    80, 96} (Nt = 64, Ls = 16, m_f = 0.05, beta = 3), nconf configurations of
    one GPU-HMC chain (the reference generator's loop, leapfrog epsilon = 0.01
    with 40 steps, mixed-CG pseudofermion solves to 1e-10, therm thermalisation
    trajectories from a seeded pure-gauge start, every configuration after them
    kept), then all their propagators -- 8 point, 16 Z4-noise and 4 wall sources
    per configuration, nconf * 28 right-hand sides -- in one dwf_measure call
    (one batched even-odd solve to 1e-10 plus every contraction), and the
    analyzer's reductions on the host. One JSON line: per Nx the HMC time and
    acceptance, the measurement's device time (CUDA events on the library
    stream, host copies included), solves/s, Schur iterations, plaquette and
    m_res."""
    import torch
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import analysis
    from three_part_dwf_study_b200.ensemble import hmc_chain, quenched_theta
    from three_part_dwf_study_b200.rng import z4_digits
    out = {"configurations_per_Nx": nconf, "rhs_per_configuration": 28, "rtol": RTOL}
    for Nx in (32, 56, 80, 96):
        Nt, Ls = 64, 16
        d = T.DomainWall(Nt, Nx, Ls, M5, MF, BETA)
        th0 = quenched_theta(np.random.default_rng(GAUGE_SEED + Nx), Nt, Nx, BETA)
        t0 = time.perf_counter()
        cfg, hist = hmc_chain(d, th0, therm + nconf, seed=GAUGE_SEED + 17 * Nx, epsilon=HMC_EPS,
                              steps=HMC_STEPS, rtol=RTOL, maxiter=MAXITER, solver=T.SOLVER_MIXED,
                              thermalization_cut=therm)
        hmc_s = time.perf_counter() - t0
        z4 = np.concatenate([z4_digits(NOISE_SEED + 104729 * k, N_NOISE * Nt * Nx * 2)
                             for k in range(nconf)])
        kw = dict(z4=z4, n_point_times=4, n_wall_times=2, n_noise=N_NOISE, max_momentum=5,
                  rtol=RTOL, maxiter=MAXITER, solver=T.SOLVER_EO_MIXED)
        st = torch.cuda.ExternalStream(d.stream_ptr())
        n_cl = d.solver_kernel_ms(2)[1]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        m = d.measure(cfg, **kw)
        e1.record(st)
        e1.synchronize()
        sec = e0.elapsed_time(e1) * 1e-3
        if not all(i["converged"] for i in m["info"]):
            raise SystemExit(f"analysis study: a solve did not converge (Nx={Nx})")
        red = analysis.reduce_ensemble(m, Nt, Nx, 2)
        nr = len(m["info"])
        out[f"64x{Nx}x16"] = {
            "hmc_seconds": sig(hmc_s), "hmc_trajectories": therm + nconf,
            "acceptance": sig(float(hist["accepted"].mean())),
            "plaquette_mean": sig(float(hist["plaquette"][therm:].mean())),
            "rhs": nr, "measure_seconds": sig(sec), "solves_per_s": sig(nr / sec),
            "ms_per_configuration": sig(1e3 * sec / nconf),
            "schur_iterations_mean": sig(statistics.mean(i["schur_iterations"] for i in m["info"])),
            "eo_kernel": "cluster" if d.solver_kernel_ms(2)[1] > n_cl else "grid",
            "m_res": sig(red["m_res_average"])}
        d.close()
    print(json.dumps({"analysis_study": out}))
    return 0


# DWF 128x128, Ls = 24, M5 = 1, m_f = 0.02, beta = 4: the larger HMC comparison
C5_LATTICE, C5_M5, C5_MF, C5_BETA = (128, 128, 24), 1.0, 0.02, 4.0


def c5_study(ntraj=200, therm=40, thin=4):
    """The study's full form at C5 size (DWF 128x128, Ls = 24, M5 = 1,
    m_f = 0.02, beta = 4): a GPU-HMC chain of ntraj trajectories from a seeded
    pure-gauge start (the reference generator's loop, epsilon = 0.01, 40
    leapfrog steps, mixed-CG pseudofermion solves to 1e-10), the configurations
    from `therm` on, every `thin`-th kept; all their propagators (28 boundary
    sources per configuration) in one dwf_measure call on the even-odd solver
    with every contraction and the analyzer's reductions; then the learned
    preconditioner trained on the first four kept configurations and used on
    the 28 sources of the fifth (flexible GCR restarted every 4 and every 16
    iterations), beside the even-odd and plain FP64 solvers on the same
    sources (all to the FP64 true residual 1e-10). One JSON line."""
    import torch
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import analysis
    from three_part_dwf_study_b200.ensemble import hmc_chain, quenched_theta
    from three_part_dwf_study_b200.rng import z4_digits
    Nt, Nx, Ls = C5_LATTICE
    d = T.DomainWall(Nt, Nx, Ls, C5_M5, C5_MF, C5_BETA)
    st = torch.cuda.ExternalStream(d.stream_ptr())
    th0 = quenched_theta(np.random.default_rng(GAUGE_SEED + 5), Nt, Nx, C5_BETA)
    t0 = time.perf_counter()
    cfg, hist = hmc_chain(d, th0, ntraj, seed=4321, epsilon=HMC_EPS, steps=HMC_STEPS, rtol=RTOL,
                          maxiter=50000, solver=T.SOLVER_MIXED, thermalization_cut=therm, thin=thin)
    hmc_s = time.perf_counter() - t0
    out = {"lattice": [Nt, Nx, Ls], "M5": C5_M5, "mf": C5_MF, "beta": C5_BETA, "trajectories": ntraj,
           "epsilon": HMC_EPS, "leapfrog_steps": HMC_STEPS, "rtol": RTOL,
           "hmc_seconds_per_trajectory": sig(hmc_s / ntraj),
           "acceptance": sig(float(hist["accepted"].mean())),
           "plaquette_mean_after_thermalisation": sig(float(hist["plaquette"][therm:].mean())),
           "plaquette_std_after_thermalisation": sig(float(hist["plaquette"][therm:].std())),
           "max_abs_dH": sig(float(np.abs(hist["dH"]).max())), "configurations_kept": len(cfg)}

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        r = fn()
        e1.record(st)
        e1.synchronize()
        return r, e0.elapsed_time(e1) * 1e-3

    # the kept configurations in calls of 8 (224 right-hand sides per call: the
    # solver's workspace for all of them at once would not fit the device)
    nconf = len(cfg)
    parts, sec = [], 0.0
    for c0 in range(0, nconf, 8):
        blk = cfg[c0:c0 + 8]
        z4 = np.concatenate([z4_digits(NOISE_SEED + 104729 * k, N_NOISE * Nt * Nx * 2)
                             for k in range(c0, c0 + len(blk))])
        kw = dict(z4=z4, n_point_times=4, n_wall_times=2, n_noise=N_NOISE, max_momentum=5, rtol=RTOL,
                  maxiter=50000, solver=T.SOLVER_EO_MIXED)
        mb, sb = timed(lambda: d.measure(blk, **kw))
        parts.append(mb)
        sec += sb
    m = {k: np.concatenate([p[k] for p in parts]) for k in ("cpp", "cj5", "loop", "mom_cpp")}
    m["info"] = [i for p in parts for i in p["info"]]
    if not all(i["converged"] for i in m["info"]):
        raise SystemExit("C5 study: a measurement solve did not converge")
    red = analysis.reduce_ensemble(m, Nt, Nx, 2)
    nr = len(m["info"])
    out["measurement"] = {"rhs": nr, "configurations_per_call": 8, "seconds": sig(sec),
                          "solves_per_s": sig(nr / sec),
                          "ms_per_configuration": sig(1e3 * sec / nconf),
                          "schur_iterations_mean": sig(statistics.mean(i["schur_iterations"] for i in m["info"])),
                          "m_res": sig(red["m_res_average"])}
    # learned preconditioner on the chain's own configurations
    d.set_gauge(np.stack(cfg[:4]))
    d.lp_init(hidden=LP_HIDDEN, seed=5)
    t0 = time.perf_counter()
    d.lp_train(**LP_TRAIN)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    d.set_gauge(cfg[4])
    src = torch.from_numpy(boundary_source_set(Nt, Nx, Ls, NOISE_SEED).view(np.float64).copy()).cuda()
    x = torch.zeros_like(src)
    res = {}
    for name, sv, restart in (("learned", T.SOLVER_LEARNED, 4), ("learned_gcr16", T.SOLVER_LEARNED, 16),
                              ("even_odd_mixed", T.SOLVER_EO_MIXED, 4),
                              ("plain_fp64_cg", T.SOLVER_CG64, 4)):
        d.lp_set_krylov(T.LP_GCR, restart)
        d.propagators_dev(src, x, rtol=RTOL, maxiter=50000, solver=sv)  # warm-up (tuning)
        infos, sec = timed(lambda: d.propagators_dev(src, x, rtol=RTOL, maxiter=50000, solver=sv))
        if not all(i["converged"] and i["true_relres"] <= RTOL * 1.0001 for i in infos):
            raise SystemExit(f"C5 study: {name} solve did not reach the FP64 true residual")
        res[name] = {"solves_per_s": sig(src.shape[0] / sec),
                     "iterations_mean": sig(statistics.mean(
                         (i["schur_iterations"] if sv != T.SOLVER_CG64 else i["iterations"]) for i in infos)),
                     "fallbacks": sum(i["fallback"] for i in infos)}
    res["learned_training_s"] = sig(train_s)
    res["learned_speedup_vs_plain_fp64"] = sig(res["learned"]["solves_per_s"] / res["plain_fp64_cg"]["solves_per_s"])
    res["even_odd_speedup_vs_plain_fp64"] = sig(res["even_odd_mixed"]["solves_per_s"]
                                                / res["plain_fp64_cg"]["solves_per_s"])
    out["propagators_28_sources"] = res
    d.close()
    print(json.dumps({"c5_study": out}))
    return 0


def hmc_compare_large(T, local, ntraj):
    """The same FP64-vs-mixed HMC comparison on DWF 128x128, Ls = 24,
    m_f = 0.02 from a seeded beta = 4 start (a bounded sample of trajectories;
    the study runs 200)."""
    from three_part_dwf_study_b200.ensemble import quenched_theta
    if ntraj < 1:
        return None
    Nt, Nx, Ls = C5_LATTICE
    d = T.DomainWall(Nt, Nx, Ls, C5_M5, C5_MF, C5_BETA, device=local)
    theta = quenched_theta(np.random.default_rng(GAUGE_SEED + 5), Nt, Nx, C5_BETA)
    try:
        res = hmc_compare(T, d, 0, ntraj, theta=theta, lattice=C5_LATTICE, seed=4321,
                          maxiter=50000)
        res.update({"M5": C5_M5, "mf": C5_MF, "beta": C5_BETA})
        return res
    finally:
        d.close()


def wilson_learned_grid(T, ntrain=8):
    """Wilson 64x64 near the critical mass: the learned preconditioner (4
    layers, 8 hidden complex channels) trained on ntrain configurations of a
    GPU Wilson-HMC chain per (beta, m0), then 16 point-source propagator solves
    to 1e-10 on the chain's next configuration, against the plain FP64 CG (CGNR) and the mixed CG
    on the same GPU. Device time per batch (CUDA events on the library
    stream, host copies of sources and solutions included), iterations and
    operator applications."""
    import torch
    from three_part_dwf_study_b200.ensemble import quenched_theta, wilson_hmc_chain
    L = 64
    out = {"lattice": [L, L], "hidden": 8, "sources": 16, "rtol": RTOL,
           "configurations": "Wilson HMC chain per setting (trajectory length 0.1 in 20 steps, CG to "
                             "1e-10) from a pure-gauge start: 10 thermalisation trajectories, then "
                             f"{ntrain} training configurations and one held out", "settings": {}}
    for beta in (2.0, 3.0, 4.0, 6.0):
        for m0 in (-0.05, 0.05):
            w = T.Wilson(L, L, m0, beta)
            st = torch.cuda.ExternalStream(w.stream_ptr())
            th0 = quenched_theta(np.random.default_rng(GAUGE_SEED + int(10 * beta)), L, L, beta)
            cfg, hist = wilson_hmc_chain(w, th0, 10 + ntrain + 1, seed=GAUGE_SEED + int(100 * (beta + m0)),
                                         epsilon=0.1 / 20, steps=20, tolerance=RTOL, max_iterations=50000,
                                         solver=T.SOLVER_MIXED, thermalization_cut=10)
            w.set_gauge(cfg[:ntrain])
            w.lp_init(hidden=8, seed=1)
            tinfo = w.lp_train(steps=3000, batch=8, lr=3e-3, lr_decay_steps=1000, pairs_per_conf=32,
                               solver_iters=50, solver_every=2, seed=3)
            w.set_gauge(cfg[ntrain])
            src = np.zeros((16, w.Ndof), np.complex128)
            for k in range(16):
                src[k, ((4 * k) * L) * 2 + (k % 2)] = 1.0
            row = {"training_loss": tinfo["loss_last"], "hmc_acceptance": float(hist["accepted"].mean())}
            for name, sv in (("learned", T.SOLVER_LEARNED), ("plain_fp64_cg", T.SOLVER_CG64),
                             ("mixed_cg", T.SOLVER_MIXED)):
                w.propagators(src, rtol=RTOL, maxiter=50000, solver=sv)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(st)
                _, infos = w.propagators(src, rtol=RTOL, maxiter=50000, solver=sv)
                e1.record(st)
                e1.synchronize()
                if not all(i["converged"] for i in infos):
                    raise SystemExit(f"Wilson solve did not converge: {name} beta={beta} m={m0}")
                it = statistics.mean(i["schur_iterations"] if sv == T.SOLVER_LEARNED else i["iterations"]
                                     for i in infos)
                # D applications: one per GCR iteration, two (D, D^dag) per CGNR iteration
                row[name] = {"ms_per_batch": e0.elapsed_time(e1), "iterations_mean": it,
                             "operator_applications_mean": (1 if sv == T.SOLVER_LEARNED else 2) * it}
            row["operator_application_ratio_plain_over_learned"] = \
                row["plain_fp64_cg"]["operator_applications_mean"] / row["learned"]["operator_applications_mean"]
            row["time_ratio_plain_over_learned"] = \
                row["plain_fp64_cg"]["ms_per_batch"] / row["learned"]["ms_per_batch"]
            out["settings"][f"beta={beta},m={m0}"] = row
            w.close()
    return out


WILSON_DSLASH_LATTICE = (2048, 2048)


def wilson_dslash(T, local, dev, peak):
    """Standalone Wilson D at 2048x2048 (working set ~400 MB >> L2) in complex128
    and complex64: V*(2*4w + 2*2w) bytes per application (spinor in and out,
    two complex links), 96 B (FP64) / 48 B (FP32) per site; the autotuned
    kernel, 20 back-to-back applications timed with CUDA events."""
    import torch
    Nt, Nx = WILSON_DSLASH_LATTICE
    w = T.Wilson(Nt, Nx, 0.1, 0.0, device=local)
    w.set_gauge(np.random.default_rng(4).uniform(-np.pi, np.pi, 2 * Nt * Nx))
    st = torch.cuda.ExternalStream(w.stream_ptr(), device=dev)
    out = {"lattice": [Nt, Nx], "bytes_rule": "V*96 B (FP64), V*48 B (FP32) per application"}
    for prec, dt, wb in ((64, torch.float64, 8), (32, torch.float32, 4)):
        a = torch.randn(w.Ndof * 2, dtype=dt, device=dev)
        b = torch.empty_like(a)
        for _ in range(3):
            w.apply_dev(0, a, b)
        w.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(20):
            w.apply_dev(0, a, b)
        e1.record(st)
        e1.synchronize()
        tsec = e0.elapsed_time(e1) * 1e-3 / 20
        gbs = Nt * Nx * (2 * 4 * wb + 2 * 2 * wb) / tsec / 1e9
        out[f"complex{2 * prec}"] = {"GBs": round(gbs, 1), "frac": round(gbs / peak, 4),
                                     "us_per_apply": round(tsec * 1e6, 2),
                                     "kernel_variant": w.dslash_variant(prec, 1)}
    w.close()
    return out


def workload_config(solver):
    return {
        "workload": (f"DWF propagator solves, {NT}x{NX} Ls={LS} M5={M5} mf={MF}, GPU-HMC beta=3.0 "
                     f"configuration, 28 boundary sources per step (8 point, 16 Z4 noise, 4 wall), "
                     f"to FP64 true residual {RTOL:g} of D^dag D"),
        "lattice": [NT, NX, LS], "rhs_per_step": 28, "rtol": RTOL, "solver": solver,
        "l2": "flushed between steps (256 MiB write)",
    }


def impl_ours(args):
    import torch
    ws, rank, local = dist_setup()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    import three_part_dwf_study_b200 as T

    dev = torch.device("cuda", local)
    d = T.DomainWall(NT, NX, LS, M5, MF, BETA, device=local)
    theta = workload_gauge(rank)
    d.set_gauge(theta)
    srcs = workload_sources(rank)
    nrhs = srcs.shape[0]
    src_dev = torch.from_numpy(srcs.view(np.float64).copy()).to(dev)
    x_dev = torch.zeros_like(src_dev)
    stream = torch.cuda.ExternalStream(d.stream_ptr(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(fn, steps, warmup, kind):
        # kind 1 is the even-odd solve (either kernel); kind 2 counts the cluster kernel alone
        for _ in range(warmup):
            fn()
        barrier()
        total = 0.0
        k0, n0 = d.solver_kernel_ms(kind)
        l0 = d.launch_count()
        infos_all = []
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            infos_all.append(fn())
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1) * 1e-3
        barrier()
        k1, n1 = d.solver_kernel_ms(kind)
        return total, infos_all, (k1 - k0) * 1e-3, n1 - n0, d.launch_count() - l0

    def step_eo():
        return d.propagators_dev(src_dev, x_dev, rtol=RTOL, maxiter=MAXITER,
                                 solver=T.SOLVER_EO_MIXED)

    def step_mixed():
        return d.propagators_dev(src_dev, x_dev, rtol=RTOL, maxiter=MAXITER,
                                 solver=T.SOLVER_MIXED)

    def step_fp64():
        return d.propagators_dev(src_dev, x_dev, rtol=RTOL, maxiter=MAXITER,
                                 solver=T.SOLVER_CG64)

    def step_learned():
        return d.propagators_dev(src_dev, x_dev, rtol=RTOL, maxiter=MAXITER,
                                 solver=T.SOLVER_LEARNED)

    # learned preconditioner: trained on four other configurations of the
    # ensemble (training time reported apart), then used on the workload one
    d.set_gauge(training_gauges(rank))
    d.lp_init(hidden=LP_HIDDEN, seed=5 + rank)
    torch.cuda.synchronize(dev)
    tt0 = time.perf_counter()
    train_info = d.lp_train(**LP_TRAIN)
    torch.cuda.synchronize(dev)
    train_s = time.perf_counter() - tt0
    d.set_gauge(theta)

    with ClockSampler(local) as clk:
        t_mixed, infos_m, kern_s, nkern, launches_eo = timed(step_eo, args.steps, args.warmup, 1)
        t_learn, infos_l, _, _, launches_l = timed(step_learned, args.steps, args.warmup, 0)
    clocks = clk.summary()
    n_side = max(1, args.steps // 2)
    t_fp64, infos_f, kern64_s, nkern64, _ = timed(step_fp64, n_side, 1, 0)
    t_full, infos_full, _, _, _ = timed(step_mixed, n_side, 1, 0)
    net_ms, net_flops = d.lp_time_network(nrhs, 10)

    for infos in infos_m + infos_f + infos_full + infos_l:
        for i in infos:
            if not i["converged"] or i["true_relres"] > RTOL * 1.0001:
                raise SystemExit(f"solve did not reach the FP64 true residual: {i}")

    # max over ranks of device time
    def allmax(v):
        if ws == 1:
            return v
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t_eo_max = allmax(t_mixed)
    t_learn_max = allmax(t_learn)
    t_fp64_max = allmax(t_fp64)
    eo_value = ws * nrhs * args.steps / t_eo_max
    learned_value = ws * nrhs * args.steps / t_learn_max
    fp64_value = ws * nrhs * n_side / t_fp64_max
    full_value = ws * nrhs * n_side / allmax(t_full)
    # the headline is the faster solver (decided by the max-over-ranks times,
    # identical on every rank)
    use_learned = learned_value > eo_value
    value = learned_value if use_learned else eo_value
    t_mixed_max = t_learn_max if use_learned else t_eo_max
    launches = launches_l if use_learned else launches_eo
    head_solver = T.SOLVER_LEARNED if use_learned else T.SOLVER_EO_MIXED

    # ---- end to end through the host C ABI ----
    src_host = torch.from_numpy(srcs.view(np.float64).copy()).pin_memory()
    x_host = torch.empty_like(src_host).pin_memory()
    th_host = torch.from_numpy(theta.copy()).pin_memory()
    src_np = src_host.numpy().view(np.complex128)
    x_np = x_host.numpy().view(np.complex128)
    th_np = th_host.numpy()

    import ctypes as C
    from three_part_dwf_study_b200 import _capi as A

    def e2e_step():
        A.check(A.lib().dwf_set_gauge(d.handle, 1, C.c_void_p(th_np.ctypes.data)), d.handle)
        infos = (A.SolveInfo * nrhs)()
        A.check(A.lib().dwf_propagators(d.handle, nrhs, None, C.c_void_p(src_np.ctypes.data),
                                        C.c_void_p(x_np.ctypes.data), RTOL, MAXITER,
                                        head_solver, infos), d.handle)
        return infos

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e2e_total = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_total += e0.elapsed_time(e1) * 1e-3
    barrier()
    e2e_value = ws * nrhs * args.steps / allmax(e2e_total)
    ref_x = x_dev.cpu().numpy().view(np.complex128)
    e2e_agree = float(np.linalg.norm(x_np - ref_x) / np.linalg.norm(ref_x))

    # ---- standalone Dslash (working set >> L2) ----
    dslash = {}
    peak, peak_kind = measured_peaks()
    Dt, Dx, Dl = DSLASH_LATTICE
    dd = T.DomainWall(Dt, Dx, Dl, M5, MF, BETA, device=local)
    dd.set_gauge(np.random.default_rng(3).uniform(-np.pi, np.pi, 2 * Dt * Dx))
    dstream = torch.cuda.ExternalStream(dd.stream_ptr(), device=dev)
    for prec, dt, w in ((64, torch.float64, 8), (32, torch.float32, 4)):
        a = torch.randn(dd.Ndof * 2, dtype=dt, device=dev)
        b = torch.empty_like(a)
        for _ in range(3):
            dd.apply_dev(0, a, b)
        dd.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record(dstream)
        for _ in range(reps):
            dd.apply_dev(0, a, b)
        e1.record(dstream)
        e1.synchronize()
        tsec = e0.elapsed_time(e1) * 1e-3 / reps
        gbs = dslash_bytes(Dt * Dx, Dl, w) / tsec / 1e9
        dslash[f"complex{2 * prec}"] = {"GBs": round(gbs, 1), "frac": round(gbs / peak, 4),
                                         "us_per_apply": round(tsec * 1e6, 2),
                                         "kernel_variant": dd.dslash_variant(prec, 1)}
    dslash["lattice"] = list(DSLASH_LATTICE)
    dslash["bytes_rule"] = "V*(Ls*64+32) B (FP64), V*(Ls*32+16) B (FP32) per application"
    dd.close()
    dslash["wilson"] = wilson_dslash(T, local, dev, peak)

    # ---- HMC on the same lattice: FP64 and mixed CG on the same trajectories ----
    hmc = hmc_compare(T, d, rank, args.hmc_trajectories)
    hmc_large = hmc_compare_large(T, local, args.hmc_large_trajectories) if ws == 1 else None
    analysis = analysis_batches(T, local) if (args.analysis and ws == 1) else None
    # ---- Wilson 64x64 near the critical mass with the learned preconditioner ----
    wil = wilson_learned_grid(T) if (args.wilson_learned and ws == 1) else None

    # ---- roofline of the dominant kernel (the persistent even-odd solver) ----
    eo_kernel_name = ("cg_eo_cluster_kernel (one thread-block cluster per right-hand side)"
                      if d.solver_kernel_ms(2)[1] > 0 else "cg_eo_mixed_kernel")
    V = NT * NX
    iters = sum(i["schur_iterations"] for infos in infos_m for i in infos)
    rus = sum(i["reliable_updates"] for infos in infos_m for i in infos)
    alg_bytes = iters * eo_iter_bytes(V, LS) + rus * eo_reliable_update_bytes(V, LS)
    kernel_launch_s = kern_s / max(1, nkern)
    achieved = alg_bytes / max(1, nkern) / kernel_launch_s / 1e9
    traffic = None
    tfile = REPO / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(
            "cg_eo_cluster_kernel_bytes_per_launch" if eo_kernel_name.startswith("cg_eo_cluster")
            else "cg_eo_mixed_kernel_bytes_per_launch")
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": eo_kernel_name, "peak_kind": f"{peak_kind} hbm_gbs (burst)",
                "alg_bytes_per_launch": alg_bytes / max(1, nkern),
                "kernel_ms_per_launch": kernel_launch_s * 1e3,
                "kernel_share_of_step": kern_s / t_mixed}

    if use_learned:
        # the dominant kernel is then the tensor-core network layer
        tpeak = measured_tensor_peak()
        ach = net_flops / (net_ms * 1e-3) / 1e12
        roofline = {"bound": "tensor", "achieved": round(ach, 1), "peak": tpeak, "unit": "TFLOP/s",
                    "frac": round(ach / tpeak, 4), "traffic": None,
                    "kernel": "lp_tc_kernel (4 launches per network application)",
                    "peak_kind": "measured bf16_tflops (burst)",
                    "alg_flops_per_application": net_flops,
                    "kernel_ms_per_application": net_ms}

    # The printed line stays short (the last few KB of output are what a log
    # tail keeps): the headline keys first, then the evidence for the two
    # targets (>= 3x plain FP64 CG; Dslash >= 70 % of HBM) at the end.
    l_iters = [i["schur_iterations"] for infos in infos_l for i in infos]
    line = {
        "metric": "dwf_propagator_solves_per_s_true_res_1e-10",
        "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed_max / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": ("bf16 network + f32 flexible GCR + f64 defect correction" if use_learned else
                  "f32+f64 (FP32 inner CG, FP64 reliable updates and true residual)"),
        "data": "synthetic (beta=3.0 configuration thermalised by the GPU HMC, boundary point/Z4/wall sources)",
        "config": dict(workload_config(
            "learned-preconditioned flexible GCR(4), FP32 inner, FP64 defect correction" if use_learned else
            "even-odd Schur mixed FP32/FP64 CG, then the full D^dag D check"),
            parallelism=f"dp{ws} (independent configurations per rank)"),
        "gpu_launches": launches,
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": "solves/s",
                "h2d_bytes_per_step": int(src_np.nbytes + th_np.nbytes),
                "d2h_bytes_per_step": int(x_np.nbytes),
                "agrees_with_device_run": sig(e2e_agree)},
        "roofline": roofline,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cs = cpu_sample(os.cpu_count() or 1)
        line["cpu_baseline"] = None if cs is None else {
            "value": cs[0], "unit": "solves/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": cs[1]}
        if REF_BENCH.exists():
            dslash["cpu_reference_apply_D"] = cpu_apply_gbs(DSLASH_LATTICE, 2)
    if hmc:
        line["hmc_64x64x16"] = {k: hmc[k] for k in ("epsilon", "leapfrog_steps", "trajectories")}
        line["hmc_64x64x16"].update(
            s_per_traj_fp64=sig(hmc["plain_fp64_cg"]["seconds_per_trajectory"]),
            s_per_traj_mixed=sig(hmc["mixed_cg"]["seconds_per_trajectory"]),
            max_abs_dH_diff=sig(hmc["max_abs_dH_difference"]))
    if hmc_large:
        line["hmc_128x128x24"] = {
            "trajectories": hmc_large["trajectories"],
            "s_per_traj_fp64": sig(hmc_large["plain_fp64_cg"]["seconds_per_trajectory"]),
            "s_per_traj_mixed": sig(hmc_large["mixed_cg"]["seconds_per_trajectory"]),
            "max_abs_dH_diff": sig(hmc_large["max_abs_dH_difference"])}
    if analysis:
        line["analysis_batched"] = {k: {"solves_per_s": sig(v["solves_per_s"]),
                                        "ms_per_conf": sig(1e3 * v["seconds_per_configuration"]),
                                        "rhs": v["rhs"]} for k, v in analysis.items()}
    if wil:
        line["learned_wilson_64x64"] = {
            k: [sig(r["time_ratio_plain_over_learned"]),
                sig(r["operator_application_ratio_plain_over_learned"])]
            for k, r in wil["settings"].items()}
        line["learned_wilson_64x64_columns"] = "time plain/learned, operator applications plain/learned"
    line["dslash"] = {
        "lattice": list(DSLASH_LATTICE),
        "complex128": dslash["complex128"], "complex64": dslash["complex64"],
        "wilson_2048x2048": {k: dslash["wilson"][k] for k in ("complex128", "complex64")}}
    if "cpu_reference_apply_D" in dslash:
        line["dslash"]["cpu_reference_apply_D"] = dslash["cpu_reference_apply_D"]
    line["learned_mixed"] = {
        "value": sig(learned_value), "speedup_vs_plain_fp64": sig(learned_value / fp64_value),
        "gcr_iterations_mean": sig(statistics.mean(l_iters)),
        "fallbacks": sum(i["fallback"] for infos in infos_l for i in infos),
        "network_ms": sig(net_ms), "network_tflops": sig(net_flops / (net_ms * 1e-3) / 1e12),
        "training_s": sig(train_s)}
    line["even_odd_mixed_cg"] = {"value": sig(eo_value),
                                 "speedup_vs_plain_fp64": sig(eo_value / fp64_value),
                                 "schur_iterations_mean": sig(statistics.mean(
                                     i["schur_iterations"] for infos in infos_m for i in infos))}
    line["plain_fp64_cg"] = {"value": sig(fp64_value), "iterations_mean": sig(statistics.mean(
        i["iterations"] for infos in infos_f for i in infos))}
    line["mixed_full_lattice_cg"] = {"value": sig(full_value)}
    if args.details and rank == 0:
        Path(args.details).write_text(json.dumps({
            "hmc": hmc, "hmc_128x128x24": hmc_large, "analysis_batched": analysis,
            "learned_wilson_64x64": wil, "dslash": dslash,
            "learned_training": dict(train_info, wall_seconds=train_s, settings=LP_TRAIN)},
            indent=1))
    if rank == 0:
        print(json.dumps(line))
    d.close()
    dd.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def profile_case():
    """One even-odd, one full-lattice mixed and one FP64 propagator batch of the
    workload (for ncu)."""
    import torch
    import three_part_dwf_study_b200 as T
    d = T.DomainWall(NT, NX, LS, M5, MF, BETA)
    d.set_gauge(workload_gauge(0))
    src = torch.from_numpy(workload_sources(0).view(np.float64).copy()).cuda()
    x = torch.zeros_like(src)
    for solver in (T.SOLVER_EO_MIXED, T.SOLVER_MIXED, T.SOLVER_CG64):
        infos = d.propagators_dev(src, x, rtol=RTOL, maxiter=MAXITER, solver=solver)
        assert all(i["converged"] for i in infos)
    d.close()
    return 0


def profile_learned():
    """The bench's training run on the training configurations, one learned
    propagator batch of the workload outside any range (kernel choices fixed
    beforehand as the bench's autotuners pick them: the tcgen05 layer kernel,
    the column-shuffle Dslash, so ncu's serialised launches cannot sway them),
    then (inside the NVTX range "learned") the same batch again and three
    network applications on 28 fields (for ncu launch lists and captures of
    the network layer kernel)."""
    import torch
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import _capi as A
    d = T.DomainWall(NT, NX, LS, M5, MF, BETA)
    d.set_gauge(training_gauges(0))
    d.lp_init(hidden=LP_HIDDEN, seed=5)
    d.lp_set_variant(1)
    A.check(A.lib().dwf_set_dslash_variant(d.handle, 5), d.handle)
    d.lp_train(**LP_TRAIN)
    d.set_gauge(workload_gauge(0))
    src = torch.from_numpy(workload_sources(0).view(np.float64).copy()).cuda()
    x = torch.zeros_like(src)
    d.propagators_dev(src, x, rtol=RTOL, maxiter=MAXITER, solver=T.SOLVER_LEARNED)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("learned")
    infos = d.propagators_dev(src, x, rtol=RTOL, maxiter=MAXITER, solver=T.SOLVER_LEARNED)
    d.lp_time_network(src.shape[0], 3)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    assert all(i["converged"] for i in infos)
    d.close()
    return 0


def profile_dslash():
    """One application of D at the Dslash bench lattice for each kernel
    variant (site, column, site with shuffled x neighbours, t sweep, column
    with shuffled x neighbours, slice ring fed by bulk copies) in FP64, then in
    FP32 (for ncu)."""
    import torch
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import _capi as A
    Dt, Dx, Dl = DSLASH_LATTICE
    d = T.DomainWall(Dt, Dx, Dl, M5, MF, BETA)
    d.set_gauge(np.random.default_rng(3).uniform(-np.pi, np.pi, 2 * Dt * Dx))
    for dt in (torch.float64, torch.float32):
        a = torch.randn(d.Ndof * 2, dtype=dt, device="cuda")
        b = torch.empty_like(a)
        for v in (0, 1, 2, 3, 5, 6):
            A.check(A.lib().dwf_set_dslash_variant(d.handle, v), d.handle)
            d.apply_dev(0, a, b)
    d.sync()
    d.close()
    return 0


def profile_wilson_dslash():
    """The Wilson operator alone at 2048x2048 (for ncu), one application per
    precision with the kernels the CUDA-event timing favours: FP64 the site
    kernel (variant 0), FP32 the t sweep at 64-row chunks (variant 3). The
    kernels are fixed rather than tuned because ncu's serialised launches
    would change the autotuner's timing."""
    import torch
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import _capi as A
    Nt, Nx = WILSON_DSLASH_LATTICE
    w = T.Wilson(Nt, Nx, 0.1, 0.0)
    w.set_gauge(np.random.default_rng(4).uniform(-np.pi, np.pi, 2 * Nt * Nx))
    for dt, v, chunk in ((torch.float64, 0, 0), (torch.float32, 3, 64)):
        A.check(A.lib().dwf_set_dslash_variant(w.handle, v), w.handle)
        A.check(A.lib().dwf_set_dslash_chunk(w.handle, chunk), w.handle)
        a = torch.randn(w.Ndof * 2, dtype=dt, device="cuda")
        b = torch.empty_like(a)
        w.apply_dev(0, a, b)
    w.sync()
    w.close()
    return 0


def profile_network():
    """Network applications only (for ncu captures of the layer kernel): the
    bench's 32-channel network with its initial weights on the workload
    configuration, applied to 28 Gaussian fields 6 times."""
    import three_part_dwf_study_b200 as T
    d = T.DomainWall(NT, NX, LS, M5, MF, BETA)
    d.set_gauge(workload_gauge(0))
    d.lp_init(hidden=LP_HIDDEN, seed=5)
    d.lp_set_variant(1)
    ms, _ = d.lp_time_network(28, 5)
    print(json.dumps({"network_ms_per_application": ms}))
    d.close()
    return 0


def eo_phases():
    """Per-phase device time of the even-odd solver kernel on one propagator
    batch of the workload (one JSON line, us per iteration)."""
    import ctypes as C
    import torch
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import _capi as A
    d = T.DomainWall(NT, NX, LS, M5, MF, BETA)
    d.set_gauge(workload_gauge(0))
    src = torch.from_numpy(workload_sources(0).view(np.float64).copy()).cuda()
    x = torch.zeros_like(src)
    d.propagators_dev(src, x, rtol=RTOL, maxiter=MAXITER, solver=T.SOLVER_EO_MIXED)  # warm-up
    A.check(A.lib().dwf_eo_phase_profile(d.handle, 1), d.handle)
    infos = d.propagators_dev(src, x, rtol=RTOL, maxiter=MAXITER, solver=T.SOLVER_EO_MIXED)
    ms = (C.c_double * 8)()
    cnt = (C.c_uint64 * 8)()
    A.check(A.lib().dwf_eo_phase_times(d.handle, ms, cnt), d.handle)
    names = ["hop_M5inv", "M5_minus_hop", "alpha_reduction", "adjoint_hop_M5inv",
             "adjoint_combine_update", "beta_reduction_reliable_updates", "direction_update"]
    out = {n: {"ms": round(ms[k], 3), "count": int(cnt[k]),
               "us_per_iteration": round(1e3 * ms[k] / max(1, cnt[k]), 2)} for k, n in enumerate(names)}
    print(json.dumps({"eo_phases": out, "schur_iterations_mean": statistics.mean(
        i["schur_iterations"] for i in infos)}))
    d.close()
    return 0


REF_GENERATE = REPO / "oracle" / "_ref" / "generate_domain_wall"
REF_ANALYZE = REPO / "oracle" / "_ref" / "analyze_domain_wall"


def ref_hmc_trajectory():
    """B4: one reference HMC trajectory (domain_wall/generate_configs.cpp,
    unmodified, one thread as the reference's generator runs) on the bench
    lattice (64x64, Ls = 16, m_f = 0.05, beta = 3, epsilon = 0.01, 40 leapfrog
    steps, pseudofermion CG to 1e-10), from the generator's own seeded start;
    wall time of the process."""
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        (d / "output" / "domain_wall").mkdir(parents=True)
        t = ref_params_text(MAXITER).replace("dwf.leapfrog_steps = 1",
                                             f"dwf.leapfrog_steps = {HMC_STEPS}")
        (d / "parameters.txt").write_text(t)
        env = dict(os.environ, OMP_NUM_THREADS="1")
        t0 = time.perf_counter()
        r = subprocess.run([str(REF_GENERATE)], cwd=d, env=env, capture_output=True, text=True,
                           timeout=7200)
        sec = time.perf_counter() - t0
        if r.returncode != 0:
            raise SystemExit(f"reference generator failed: {r.stderr.strip()[-400:]}")
    return {"seconds_per_trajectory": round(sec, 2), "threads": 1, "lattice": [NT, NX, LS],
            "epsilon": HMC_EPS, "leapfrog_steps": HMC_STEPS, "rtol": RTOL,
            "source": "domain_wall/generate_configs.cpp, one trajectory"}


def ref_analyzer(Nx=32, noise=8, nconf=None):
    """B6: the reference analyzer (domain_wall/analyze_configs.cpp, unmodified)
    on Nt = 64, Nx, Ls = 16 for nconf seeded beta = 3 configurations (default:
    as many as host threads; the first ones are the bench's `analysis_batched`
    configurations), analysis.threads = 0 (one configuration per OpenMP
    thread), propagators to 1e-10, eta.noise_vectors = noise (8, the value in
    the reference's parameters.txt): per configuration 2 x 2 wall, 2 x 2 point
    and `noise` noise solves plus the contractions; seconds per configuration =
    wall time / configurations."""
    from three_part_dwf_study_b200.ensemble import quenched_theta
    nconf = nconf or (os.cpu_count() or 1)
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        (d / "output" / "domain_wall").mkdir(parents=True)
        Nt, Ls = 64, 16
        t = ref_params_text(MAXITER, Nt, Nx, Ls).replace(
            "eta.noise_vectors = 1", f"eta.noise_vectors = {noise}").replace(
            "analysis.max_momentum = 1", "analysis.max_momentum = 5")
        (d / "parameters.txt").write_text(t)
        rng = np.random.default_rng(GAUGE_SEED + Nx)
        th = np.stack([quenched_theta(rng, Nt, Nx, BETA).reshape(2, Nt, Nx) for _ in range(nconf)])
        np.save(d / "output" / "domain_wall" / "analysis_configs.npy", th)
        t0 = time.perf_counter()
        r = subprocess.run([str(REF_ANALYZE)], cwd=d, capture_output=True, text=True, timeout=7200)
        sec = time.perf_counter() - t0
    measured = r.stdout.count("measuring config")
    if measured != nconf:
        raise SystemExit(f"reference analyzer measured {measured} of {nconf} configurations: "
                         f"{r.stderr.strip()[-400:]}")
    rhs = 4 + 4 + noise
    return {"seconds_per_configuration": round(sec / nconf, 3), "configurations": nconf,
            "threads": os.cpu_count() or 1, "wall_seconds": round(sec, 2),
            "rhs_per_configuration": rhs, "solves_per_s": round(rhs * nconf / sec, 3),
            "lattice": [Nt, Nx, Ls], "rtol": RTOL, "exit_code": r.returncode,
            "source": "domain_wall/analyze_configs.cpp, all configurations in one run"}


def cpu_reference_extras():
    """BASELINE's B4 (reference HMC trajectory) and B6 (reference analyzer per
    configuration) on the host cores, one JSON line (their GPU counterparts:
    the bench line's `hmc_64x64x16` and `analysis_batched`)."""
    if not (REF_GENERATE.exists() and REF_ANALYZE.exists()):
        print(json.dumps({"cpu_reference_extras": "unavailable: oracle/_ref executables not built"}))
        return 0
    out = {"B6_analyzer_64x32x16": ref_analyzer(32), "B4_hmc_trajectory_64x64x16": ref_hmc_trajectory()}
    print(json.dumps({"cpu_reference_extras": out}))
    return 0


def dslash_variants():
    """Event-timed GB/s of the Dslash kernels (site, column, site with shuffled
    x neighbours, t sweep at the automatic and at fixed chunk lengths, and for
    Wilson the row kernel) in FP64
    and FP32 at 256x256x16, 512x512x16 and on the 2048x2048 Wilson lattice
    (Ls = 1; one JSON line)."""
    import torch
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import _capi as A
    out = {}
    for lat in ((256, 256, 16), DSLASH_LATTICE, WILSON_DSLASH_LATTICE + (1,)):
        Dt, Dx, Dl = lat
        if Dl == 1:
            d = T.Wilson(Dt, Dx, 0.1, 0.0)
        else:
            d = T.DomainWall(Dt, Dx, Dl, M5, MF, BETA)
        d.set_gauge(np.random.default_rng(3).uniform(-np.pi, np.pi, 2 * Dt * Dx))
        st = torch.cuda.ExternalStream(d.stream_ptr())
        for prec, dt, w in ((64, torch.float64, 8), (32, torch.float32, 4)):
            a = torch.randn(d.Ndof * 2, dtype=dt, device="cuda")
            b = torch.empty_like(a)
            kinds = [(0, 0, "site"), (1, 0, "column"), (2, 0, "site_shuffle"), (5, 0, "column_shuffle"),
                     (6, 0, "slice_ring"),
                     (3, 0, "t_sweep_auto"), (3, 8, "t_sweep_8"), (3, 16, "t_sweep_16"),
                     (3, 32, "t_sweep_32"), (3, 64, "t_sweep_64")]
            if Dl == 1:
                kinds += [(3, 128, "t_sweep_128"), (3, 256, "t_sweep_256"),
                          (3, 2048, "t_sweep_2048"), (4, 0, "rows")]
            for v, chunk, name in kinds:
                A.check(A.lib().dwf_set_dslash_chunk(d.handle, chunk), d.handle)
                A.check(A.lib().dwf_set_dslash_variant(d.handle, v), d.handle)
                for _ in range(3):
                    d.apply_dev(0, a, b)
                d.sync()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                for _ in range(20):
                    d.apply_dev(0, a, b)
                e1.record(st)
                e1.synchronize()
                tsec = e0.elapsed_time(e1) * 1e-3 / 20
                tag = f"wilson_{Dt}x{Dx}" if Dl == 1 else f"{Dt}x{Dx}x{Dl}"
                out[f"{tag}_fp{prec}_{name}"] = round(dslash_bytes(Dt * Dx, Dl, w) / tsec / 1e9, 1)
        d.close()
    print(json.dumps({"dslash_GBs": out, "bytes_rule": "V*(Ls*64+32) FP64, V*(Ls*32+16) FP32; "
                      "Wilson (Ls = 1) V*96 FP64, V*48 FP32"}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--details", default=None,
                    help="also write every section's full record to this JSON file")
    ap.add_argument("--no-analysis", dest="analysis", action="store_false",
                    help="skip the batched-analyzer timing (Nt=64, Nx=32 and 96)")
    ap.add_argument("--hmc-large-trajectories", type=int, default=1,
                    help="HMC trajectories of the 128x128x24 FP64-vs-mixed comparison (0: skip)")
    ap.add_argument("--hmc-trajectories", type=int, default=2,
                    help="HMC trajectories compared between FP64 and mixed CG (0: skip)")
    ap.add_argument("--no-wilson-learned", dest="wilson_learned", action="store_false",
                    help="skip the Wilson 64x64 learned-preconditioner grid")
    ap.add_argument("--profile-case", action="store_true")
    ap.add_argument("--profile-dslash", action="store_true")
    ap.add_argument("--profile-learned", action="store_true")
    ap.add_argument("--profile-network", action="store_true")
    ap.add_argument("--profile-wilson-dslash", action="store_true")
    ap.add_argument("--dslash-variants", action="store_true")
    ap.add_argument("--eo-phases", action="store_true")
    ap.add_argument("--analysis-study", action="store_true",
                    help="64 GPU-HMC configurations per Nx in {32,56,80,96}, all propagators in one call")
    ap.add_argument("--c5-study", action="store_true",
                    help="200 GPU-HMC trajectories at 128x128x24, their analysis and the learned solver there")
    ap.add_argument("--cpu-reference-extras", action="store_true",
                    help="time the reference's own HMC trajectory (B4) and analyzer (B6) on the host cores")
    args = ap.parse_args()
    if args.cpu_reference_extras:
        return cpu_reference_extras()
    if args.c5_study:
        return c5_study()
    if args.profile_case:
        return profile_case()
    if args.profile_dslash:
        return profile_dslash()
    if args.profile_learned:
        return profile_learned()
    if args.profile_network:
        return profile_network()
    if args.profile_wilson_dslash:
        return profile_wilson_dslash()
    if args.dslash_variants:
        return dslash_variants()
    if args.eo_phases:
        return eo_phases()
    if args.analysis_study:
        return analysis_study()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return impl_reference(args)
    return impl_ours(args)


if __name__ == "__main__":
    sys.exit(main())
