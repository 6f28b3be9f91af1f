"""Seeded pure-gauge starting configurations of the 2-D U(1) theory.

In two dimensions the plaquette angles of the pure-gauge theory at coupling
beta are independent with density proportional to exp(beta cos P) (the
periodic closure ties one plaquette per time slice to the others). A
configuration is built in the axial gauge from such plaquettes and then
gauge-randomised. These serve as thermalised-like starting points of
measurement ensembles and as the training configurations of the learned
preconditioner; the dynamical-fermion HMC (DomainWall.hmc_trajectory) refines
them where the fermion determinant matters.
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
