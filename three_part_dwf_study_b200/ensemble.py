"""Seeded pure-gauge starting configurations of the 2-D U(1) theory.

In two dimensions the plaquette angles of the pure-gauge theory at coupling
beta are independent with density proportional to exp(beta cos P) (the
periodic closure ties one plaquette per time slice to the others). A
configuration is built in the axial gauge from such plaquettes and then
gauge-randomised. These serve as thermalised-like starting points of
measurement ensembles and as the training configurations of the learned
preconditioner; the dynamical-fermion HMC (DomainWall.hmc_trajectory) refines
them where the fermion determinant matters. hmc_chain runs the reference
generator's whole Markov chain (draws, leapfrog, Metropolis, thermalisation cut
and thinning) on the GPU and yields HMC-generated ensembles.
"""
import numpy as np


def quenched_theta(rng, Nt, Nx, beta):
    """Link angles theta[mu][t][x] (flat, gauge_index layout) in [-pi, pi).
    rng: numpy Generator."""
    P = rng.vonmises(0.0, beta, size=(Nt, Nx))
    th = np.zeros((2, Nt, Nx))
    th[1, 0] = rng.uniform(-np.pi, np.pi, Nx)
    for t in range(Nt - 1):
        th[1, t + 1] = th[1, t] + P[t]
    for x in range(Nx - 1):
        th[0, Nt - 1, x + 1] = th[0, Nt - 1, x] + th[1, 0, x] - th[1, Nt - 1, x] - P[Nt - 1, x]
    phi = rng.uniform(-np.pi, np.pi, (Nt, Nx))
    th[0] += phi - np.roll(phi, -1, 0)
    th[1] += phi - np.roll(phi, -1, 1)
    return np.angle(np.exp(1j * th)).ravel()


def quenched_ensemble(seed, n, Nt, Nx, beta):
    """n configurations [n][2 Nt Nx] from one seeded generator."""
    rng = np.random.default_rng(seed)
    return np.stack([quenched_theta(rng, Nt, Nx, beta) for _ in range(n)])


def hmc_chain(d, theta0, trajectories, seed, epsilon, steps, rtol=1e-10, maxiter=5000,
              solver=None, thermalization_cut=0, thin=1):
    """The domain-wall generator's Markov chain on the GPU
    (domain_wall/generate_configs.cpp:48-207): per trajectory, from one
    std::mt19937_64(seed) stream, chi (Ndof complex, imaginary part first),
    then the momenta (2 Nt Nx normals), then the Metropolis uniform; phi = D chi,
    leapfrog (DomainWall.hmc_trajectory), accept if u < min(exp(-dH), 1).
    Configurations from trajectory `thermalization_cut` on, every `thin`-th,
    are kept (the reference's analysis_configs).

    d: DomainWall context. Returns (configs [n][2 Nt Nx], history) with history
    a dict of per-trajectory arrays accepted, dH, acceptance_probability,
    plaquette (of the chain's configuration after the decision)."""
    from . import _capi as A
    from .rng import Rng

    solver = A.SOLVER_MIXED if solver is None else solver
    rng = Rng(seed)
    th = np.ascontiguousarray(theta0, dtype=np.float64).reshape(-1).copy()
    kept = []
    hist = {k: np.zeros(trajectories) for k in ("accepted", "dH", "acceptance_probability",
                                                 "plaquette")}
    for k in range(trajectories):
        chi = rng.pseudofermion(d.Ndof)
        mom = rng.normals(d.Ngauge)
        prop, info = d.hmc_trajectory(th, chi, mom, epsilon, steps, rtol=rtol, maxiter=maxiter,
                                      solver=solver)
        pacc = min(float(np.exp(-info["dH"])), 1.0)
        acc = rng.uniform() < pacc
        if acc:
            th = prop
        hist["accepted"][k] = acc
        hist["dH"][k] = info["dH"]
        hist["acceptance_probability"][k] = pacc
        hist["plaquette"][k] = d.average_plaquette(th)
        if k >= thermalization_cut and (k - thermalization_cut) % thin == 0:
            kept.append(th.copy())
    configs = np.stack(kept) if kept else np.zeros((0, d.Ngauge))
    return configs, hist


def wilson_hmc_chain(w, theta0, trajectories, seed, epsilon, steps, tolerance=1e-10,
                     max_iterations=5000, solver=None, thermalization_cut=0, thin=1):
    """A Wilson pseudofermion HMC Markov chain on the GPU: per trajectory,
    from one numpy generator seeded with `seed`, the momenta (2 Nt Nx normals),
    the pseudofermion chi (Ndof complex normals, variance 1/2 per part) and the
    Metropolis uniform, then Wilson.hmc_step (leapfrog and accept/reject,
    wilson/include/gauge.hpp:132-180). Configurations from trajectory
    `thermalization_cut` on, every `thin`-th, are kept.

    w: Wilson context. Returns (configs [n][2 Nt Nx], history) with history a
    dict of per-trajectory arrays accepted, dH, plaquette."""
    from . import _capi as A

    solver = A.SOLVER_CG64 if solver is None else solver
    rng = np.random.default_rng(seed)
    th = np.ascontiguousarray(theta0, dtype=np.float64).reshape(-1).copy()
    kept = []
    hist = {k: np.zeros(trajectories) for k in ("accepted", "dH", "plaquette")}
    for k in range(trajectories):
        mom = rng.normal(size=w.Ngauge)
        chi = (rng.normal(size=w.Ndof) + 1j * rng.normal(size=w.Ndof)) / np.sqrt(2.0)
        u = rng.uniform()
        th, info = w.hmc_step(th, mom, chi, u, epsilon, steps, tolerance, max_iterations,
                              solver=solver)
        hist["accepted"][k] = info["accepted"]
        hist["dH"][k] = info["dH"]
        hist["plaquette"][k] = w.average_plaquette(th)
        if k >= thermalization_cut and (k - thermalization_cut) % thin == 0:
            kept.append(th.copy())
    configs = np.stack(kept) if kept else np.zeros((0, w.Ngauge))
    return configs, hist
