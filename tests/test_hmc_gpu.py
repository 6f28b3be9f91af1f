"""HMC pieces and whole trajectories on the GPU against the oracle and the
reference's golden outputs (domain wall and Wilson).

Tolerances: at the reference's own solver tolerances (1e-12 and looser) the
golden solutions and forces carry the CG truncation error, so they are
compared at 1e-10; with both sides solving to rtol 1e-14 (where the oracle's
CG is within 5e-14 of a dense direct solve, tests/test_oracle_golden.py) the
FP64 solutions, pseudofermion forces and actions agree within 1e-12 relative.
Per-trajectory dH within 1e-7 absolute; configurations after a trajectory
within 1e-9 relative; accept/reject decisions identical to the reference's
own runs."""
import csv

import numpy as np
import pytest

from conftest import random_field, random_theta, rel
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import three_part_dwf_study_b200 as T
    return T


def test_gauge_action_force_plaquette(T, golden):
    for case in ["dwf_8x8x4", "dwf_6x10x3"]:
        g = golden(case)
        p = g.p
        d = T.DomainWall(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"],
                         p["dwf.beta"])
        th = g.npy("in_theta.npy")
        a, f = d.gauge_action_force(th)
        info = g.npy("out_gauge_info.npy")
        assert abs(a - info[0]) < 1e-12 * abs(info[0])
        assert rel(f, g.npy("out_gauge_force.npy")) < 1e-13
        assert abs(d.average_plaquette(th) - info[1]) < 1e-14


@pytest.mark.parametrize("case", ["dwf_8x8x4", "dwf_6x10x3"])
def test_pseudofermion_action_force_golden(T, golden, case):
    g = golden(case)
    p = g.p
    d = T.DomainWall(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"],
                     p["dwf.beta"])
    th, chi = g.npy("in_theta.npy"), g.field("in_chi.npy")
    phi = d.apply_D(th, chi)
    pf = d.pseudofermion_action_force(th, phi, rtol=p["dwf.pseudofermion_rtol"],
                                      maxiter=p["dwf.pseudofermion_maxiter"])
    info = g.npy("out_pf_info.npy")
    assert abs(pf["action"] - info[0]) < 1e-11 * abs(info[0])
    assert abs(pf["iterations"] - info[1]) <= 2
    assert rel(pf["force"], g.npy("out_pf_force.npy")) < 1e-10
    assert rel(pf["eta"], g.field("out_pf_eta.npy")) < 1e-10
    warm = d.pseudofermion_action_force(th, phi, eta_guess=pf["eta"],
                                        rtol=p["dwf.pseudofermion_rtol"],
                                        maxiter=p["dwf.pseudofermion_maxiter"])
    assert abs(warm["iterations"] - g.npy("out_pf_warm_info.npy")[1]) <= 2


@pytest.mark.parametrize("case", ["dwf_8x8x4", "dwf_6x10x3"])
def test_pseudofermion_action_force_within_1e12(T, golden, case):
    """eta = (D D^dag)^-1 phi, S = Re<phi, eta> and the force against the oracle
    (domain_wall/include/pseudofermion.hpp:22-166), both solving to rtol 1e-14;
    cold start and the HMC's warm start from a nearby eta."""
    g = golden(case)
    p = g.p
    d = T.DomainWall(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"],
                     p["dwf.beta"])
    o = O.Dwf(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"])
    th = g.npy("in_theta.npy")
    phi = o.apply(0, th, g.field("in_chi.npy"))
    guess = None
    for start in ("cold", "warm"):
        pf = d.pseudofermion_action_force(th, phi, eta_guess=guess, rtol=1e-14, maxiter=20000)
        ref = o.pf_action_force(th, phi, 1e-14, 20000, guess=guess)
        assert ref["status"] == 0
        assert rel(pf["eta"], ref["eta"]) < 1e-12, start
        assert rel(pf["force"], ref["force"]) < 1e-12, start
        assert abs(pf["action"] - ref["action"]) < 1e-12 * abs(ref["action"]), start
        assert abs(pf["iterations"] - ref["iterations"]) <= 2, start
        guess = ref["eta"] * (1.0 + 1e-3 * np.cos(np.arange(ref["eta"].size)))


def test_pseudofermion_force_is_action_derivative(T):
    """F_l = dS_pf/dtheta_l (central difference, h = 1e-5)."""
    rng = np.random.default_rng(31)
    Nt, Nx, Ls = 6, 6, 4
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.2, 2.0)
    th = random_theta(rng, Nt, Nx)
    phi = random_field(rng, Ls * Nt * Nx * 2)
    F = d.pseudofermion_action_force(th, phi, rtol=1e-14, maxiter=5000)["force"]
    h = 1e-5
    for l in [0, 7, 2 * Nt * Nx - 1, Nt * Nx + 3]:
        tp, tm = th.copy(), th.copy()
        tp[l] += h
        tm[l] -= h
        sp = d.pseudofermion_action_force(tp, phi, rtol=1e-14, maxiter=5000)["action"]
        sm = d.pseudofermion_action_force(tm, phi, rtol=1e-14, maxiter=5000)["action"]
        assert abs((sp - sm) / (2 * h) - F[l]) < 1e-6 * max(1.0, abs(F[l]))


@pytest.mark.parametrize("solver", [0, 1])
def test_dwf_trajectory_matches_oracle(T, solver):
    rng = np.random.default_rng(41)
    Nt, Nx, Ls = 8, 6, 4
    beta, eps, steps = 3.0, 0.05, 6
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.1, beta)
    o = O.Dwf(Nt, Nx, Ls, 1.0, 0.1)
    th0 = random_theta(rng, Nt, Nx) * 0.3
    chi = random_field(rng, o.ndof)
    mom = rng.normal(size=o.ngauge)
    out, info = d.hmc_trajectory(th0, chi, mom, eps, steps, rtol=1e-12, maxiter=5000,
                                 solver=solver)
    st, oth, oinf = o.trajectory(beta, eps, steps, 1e-12, 5000, th0, chi, mom)
    assert st == 0
    assert abs(info["dH"] - oinf["dH"]) < 1e-7
    assert abs(info["H0"] - oinf["H0"]) < 1e-9 * abs(oinf["H0"])
    assert rel(out, oth) < 1e-9
    assert info["solves"] == steps + 1


def test_dwf_chain_reproduces_reference_generator(T, golden):
    """Four trajectories of the reference's generate_domain_wall (its RNG stream,
    seed 1234, cold start theta = 1): same decisions, same configurations."""
    g = golden("dwf_hmc_8x8x4")
    p = g.p
    d = T.DomainWall(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"],
                     p["dwf.beta"])
    cfg = g.npy("configs.npy")
    hist = list(csv.DictReader(open(g.dir / "run_info_history.csv")))
    chi, mom, u = O.dwf_draws(p["dwf.random_seed"], p["dwf.trajectories"], d.Ndof, d.Ngauge)
    th = np.ones(d.Ngauge)
    for k in range(p["dwf.trajectories"]):
        prop, info = d.hmc_trajectory(th, chi[k], mom[k], p["dwf.epsilon"],
                                      p["dwf.leapfrog_steps"], rtol=p["dwf.pseudofermion_rtol"],
                                      maxiter=p["dwf.pseudofermion_maxiter"])
        acc = u[k] < min(np.exp(-info["dH"]), 1.0)
        assert int(acc) == int(hist[k]["accepted"])
        assert float(hist[k]["delta_h"]) == pytest.approx(info["dH"], rel=1e-5, abs=1e-9)
        if acc:
            th = prop
        assert rel(th, cfg[k].ravel()) < 1e-9
        assert d.average_plaquette(th) == pytest.approx(float(hist[k]["plaquette"]), abs=1e-5)


def test_dh_scales_as_eps_squared(T):
    rng = np.random.default_rng(51)
    Nt, Nx, Ls = 8, 8, 4
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.2, 2.0)
    th0 = random_theta(rng, Nt, Nx) * 0.2
    chi = random_field(rng, d.Ndof)
    mom = rng.normal(size=d.Ngauge)
    dh = []
    for eps, steps in [(0.04, 5), (0.02, 10)]:
        _, info = d.hmc_trajectory(th0, chi, mom, eps, steps, rtol=1e-12, maxiter=5000)
        dh.append(abs(info["dH"]))
    assert 2.5 < dh[0] / dh[1] < 6.0


# ---------------------------------------------------------------------------
# Wilson
# ---------------------------------------------------------------------------
def wil_of(T, g):
    p = g.p
    return T.Wilson(p["wilson.Nt"], p["wilson.Nx"], p["wilson.m0"], p["wilson.beta"],
                    p["wilson.time_boundary_sign"], p["wilson.space_boundary_sign"])


@pytest.mark.parametrize("case", ["wil_8x8", "wil_6x10"])
def test_wilson_operators_and_solves_golden(T, golden, case):
    g = golden(case)
    p = g.p
    w = wil_of(T, g)
    th, psi = g.npy("in_theta.npy"), g.field("in_psi.npy")
    assert rel(w.apply_D(th, psi), g.field("out_D.npy")) < 1e-13
    assert rel(w.apply_D_dagger(th, psi), g.field("out_Ddag.npy")) < 1e-13
    r = w.solve_CGNR(th, psi, p["wilson.measurement_cg_tolerance"],
                     p["wilson.measurement_cg_max_iterations"])
    info = g.npy("out_cgnr_info.npy")
    assert abs(r["iterations"] - info[0]) <= 2
    assert rel(r["x"], g.field("out_cgnr_x.npy")) < 1e-10
    assert r["normal_residual"] < 20 * p["wilson.measurement_cg_tolerance"]
    assert r["dirac_residual"] == pytest.approx(info[2], rel=0.5)
    eta = w.solve_DDdag(th, psi, p["wilson.force_cg_tolerance"],
                        p["wilson.force_cg_max_iterations"])
    assert rel(eta, g.field("out_dddag_x.npy")) < 1e-10
    acts = g.npy("out_actions.npy")
    a, f = w.gauge_action_force(th)
    assert abs(a - acts[0]) < 1e-12 * abs(acts[0])
    assert rel(f, g.npy("out_gauge_force.npy")) < 1e-13
    pf = w.pseudofermion_action_force(th, psi, rtol=p["wilson.force_cg_tolerance"],
                                      maxiter=p["wilson.force_cg_max_iterations"])
    assert abs(pf["action"] - acts[1]) < 1e-10 * abs(acts[1])
    assert rel(pf["force"], g.npy("out_pf_force.npy")) < 1e-10


@pytest.mark.parametrize("case", ["wil_8x8", "wil_6x10"])
def test_wilson_solutions_and_force_within_1e12(T, golden, case):
    """solve_CGNR, solve_DDdag (wilson/include/cg_solver.hpp:19-78) and the
    pseudofermion action and force (wilson/include/gauge.hpp:68-122) against the
    oracle, both solving to tolerance 1e-14."""
    g = golden(case)
    p = g.p
    w = wil_of(T, g)
    o = O.Wilson(p["wilson.Nt"], p["wilson.Nx"], p["wilson.m0"], p["wilson.time_boundary_sign"],
                 p["wilson.space_boundary_sign"])
    th, psi = g.npy("in_theta.npy"), g.field("in_psi.npy")
    tol = 1e-14
    r = w.solve_CGNR(th, psi, tol, 20000)
    st, xo, info = o.solve_cgnr(th, psi, tol, 20000)
    assert st == 0
    assert rel(r["x"], xo) < 1e-12
    assert abs(r["iterations"] - info[0]) <= 2
    eta = w.solve_DDdag(th, psi, tol, 20000)
    st, etao, _ = o.solve_dddag(th, psi, tol, 20000)
    assert st == 0
    assert rel(eta, etao) < 1e-12
    pf = w.pseudofermion_action_force(th, psi, rtol=tol, maxiter=20000)
    st, act, force = o.pf_action_force(th, psi, tol, 20000)
    assert st == 0
    assert rel(pf["force"], force) < 1e-12
    assert abs(pf["action"] - act) < 1e-12 * abs(act)


@pytest.mark.parametrize("case", ["wil_8x8", "wil_6x10"])
def test_wilson_hmc_step_reproduces_reference(T, golden, case):
    """Three hmc_step calls with the reference's RNG stream reproduce its
    configurations, dH and decisions."""
    g = golden(case)
    p = g.p
    w = wil_of(T, g)
    mom, chi, u = O.wil_draws(p["wilson.random_seed"], 3, w.Ntot, w.Ngauge)
    thetas, info = g.npy("out_hmc_theta.npy"), g.npy("out_hmc_info.npy")
    cur = g.npy("in_theta.npy").ravel()
    eps = p["wilson.trajectory_length"] / p["wilson.hmc_steps"]
    for k in range(3):
        cur, inf = w.hmc_step(cur, mom[k], chi[k], u[k], eps, p["wilson.hmc_steps"],
                              p["wilson.force_cg_tolerance"],
                              p["wilson.force_cg_max_iterations"])
        assert abs(inf["dH"] - info[k, 0]) < 1e-8
        assert inf["accepted"] == int(info[k, 2])
        assert rel(cur, thetas[k].ravel()) < 1e-9


def test_wilson_solver_failure_reports_reference_message(T):
    rng = np.random.default_rng(61)
    w = T.Wilson(8, 8, 0.1, 2.0)
    th = random_theta(rng, 8, 8)
    with pytest.raises(RuntimeError, match="CGNR failed: iterations="):
        w.solve_CGNR(th, random_field(rng, w.Ndof), 1e-12, 3)
    with pytest.raises(RuntimeError, match="pseudofermion CG failed: iterations="):
        w.solve_DDdag(th, random_field(rng, w.Ndof), 1e-12, 3)
