"""Ensembles the GPU generates, against the reference's CPU path (the oracle).

* Wilson 32x32 HMC (beta 2, m0 0.1, hot start, tau = 1 in 20 leapfrog steps,
  FP64 CG to 1e-10, 20 trajectories; wilson/include/gauge.hpp:124-180): the GPU
  chain and the oracle's, each run on its own from the same start and the
  reference's draws (momenta, pseudofermion, uniform per trajectory), take the
  same accept/reject decisions with dH per trajectory within 1e-6 and the
  configurations within 1e-7 relative.
* Domain wall Nt = 64, Nx = 32, Ls = 16, beta 3, m_f 0.05: configurations
  thermalised by the GPU HMC chain (the reference generator's loop,
  domain_wall/generate_configs.cpp:48-207) are measured by the GPU's batched
  analyzer and by the oracle's compute_CPP_CJ5 (domain_wall/include/
  correlator.hpp:243-310) on the same configuration: C_PP, C_J5 within 1e-8
  and the residual mass ratio C_J5/C_PP (domain_wall/analyze_configs.cpp:98-113)
  within 1e-8 when both solve to 1e-12; plaquettes within 1e-14.
* Domain wall 8x8x4: two independent Markov chains of 300 trajectories, one on
  the GPU (mixed-precision pseudofermion solves) and one in the oracle (the
  reference algorithm), agree within four standard errors (13 bins) on the
  plaquette, C_PP(t) and the residual mass.
"""
import numpy as np
import pytest

from conftest import rel
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import three_part_dwf_study_b200 as T
    return T


# ---------------------------------------------------------------------------
# Wilson 32x32 chain
# ---------------------------------------------------------------------------
W_NT = W_NX = 32
W_BETA, W_M0, W_STEPS, W_NTRAJ, W_TOL = 2.0, 0.1, 20, 20, 1e-10


@pytest.fixture(scope="module")
def wilson_oracle_chain():
    w = O.Wilson(W_NT, W_NX, W_M0)
    th0 = np.random.default_rng(1234).uniform(-np.pi, np.pi, w.ngauge)
    mom, chi, u = O.wil_draws(1234, W_NTRAJ, w.ntot, w.ngauge)
    cur, hist = th0.copy(), []
    for k in range(W_NTRAJ):
        st, cur, inf = w.hmc_step(W_BETA, 1.0 / W_STEPS, W_STEPS, W_TOL, 4000, cur, mom[k],
                                  chi[k], u[k])
        assert st == 0
        hist.append((inf["dH"], inf["accepted"], cur.copy()))
    return th0, (mom, chi, u), hist


@pytest.mark.parametrize("solver", [0, 1])
def test_wilson_32x32_chain_matches_oracle(T, wilson_oracle_chain, solver):
    th0, (mom, chi, u), hist = wilson_oracle_chain
    w = T.Wilson(W_NT, W_NX, W_M0, W_BETA)
    cur = th0.copy()
    for k in range(W_NTRAJ):
        cur, inf = w.hmc_step(cur, mom[k], chi[k], u[k], 1.0 / W_STEPS, W_STEPS, W_TOL, 4000,
                              solver=solver)
        dh, acc, oth = hist[k]
        assert bool(inf["accepted"]) == bool(acc), f"trajectory {k}"
        assert abs(inf["dH"] - dh) < 1e-6, f"trajectory {k}"
        assert rel(cur, oth) < 1e-7, f"trajectory {k}"
    assert any(h[1] for h in hist)
    w.close()


def test_wilson_hmc_chain_helper_matches_oracle(T):
    """ensemble.wilson_hmc_chain (the chain that generates the Wilson
    learned-preconditioner grid's configurations): its draws replayed through
    the oracle's hmc_step give the same decisions, dH and configurations, and
    the thermalisation cut and thinning keep the right trajectories."""
    from three_part_dwf_study_b200.ensemble import wilson_hmc_chain
    Nt = Nx = 16
    beta, m0, eps, steps, ntraj = 2.0, 0.1, 0.05, 20, 6
    w = T.Wilson(Nt, Nx, m0, beta)
    th0 = np.random.default_rng(7).uniform(-np.pi, np.pi, w.Ngauge)
    cfg, hist = wilson_hmc_chain(w, th0, ntraj, seed=99, epsilon=eps, steps=steps, tolerance=1e-10,
                                 max_iterations=4000, thermalization_cut=2, thin=2)
    assert cfg.shape == (2, w.Ngauge)
    o = O.Wilson(Nt, Nx, m0)
    rng = np.random.default_rng(99)
    cur = th0.copy()
    kept = []
    for k in range(ntraj):
        mom = rng.normal(size=w.Ngauge)
        chi = (rng.normal(size=w.Ndof) + 1j * rng.normal(size=w.Ndof)) / np.sqrt(2.0)
        u = rng.uniform()
        st, cur, inf = o.hmc_step(beta, eps, steps, 1e-10, 4000, cur, mom, chi, u)
        assert st == 0
        assert bool(inf["accepted"]) == bool(hist["accepted"][k]), k
        assert abs(inf["dH"] - hist["dH"][k]) < 1e-6, k
        if k >= 2 and (k - 2) % 2 == 0:
            kept.append(cur.copy())
    for a, b in zip(cfg, kept):
        assert rel(a, b) < 1e-7
    assert np.all(np.isfinite(hist["plaquette"]))
    w.close()


# ---------------------------------------------------------------------------
# Domain wall: GPU-HMC configurations measured on both sides
# ---------------------------------------------------------------------------
def test_gpu_hmc_configuration_measured_like_reference(T):
    from three_part_dwf_study_b200.ensemble import hmc_chain

    Nt, Nx, Ls, M5, mf, beta = 64, 32, 16, 1.0, 0.05, 3.0
    d = T.DomainWall(Nt, Nx, Ls, M5, mf, beta)
    # the reference's leapfrog (dwf.epsilon 0.01, 40 steps) from a cold start
    cfg, hist = hmc_chain(d, np.zeros(d.Ngauge), 40, seed=1234, epsilon=0.01, steps=40,
                          rtol=1e-8, maxiter=5000, solver=T.SOLVER_MIXED,
                          thermalization_cut=39)
    assert hist["accepted"].sum() >= 24
    # moved away from the cold start (plaquette 1)
    assert 0.6 < hist["plaquette"][-1] < 0.97
    th = cfg[-1]
    m = d.measure(th, n_point_times=2, n_wall_times=2, n_noise=0, max_momentum=0, rtol=1e-12,
                  maxiter=20000, solver=T.SOLVER_EO_MIXED)
    assert all(i["converged"] for i in m["info"])
    o = O.Dwf(Nt, Nx, Ls, M5, mf)
    st, cpp, cj5 = o.cpp_cj5(th, 1e-12, 20000)
    assert st == 0
    assert rel(m["cpp"][0], cpp) < 1e-8
    assert rel(m["cj5"][0], cj5) < 1e-8
    assert rel(m["cj5"][0] / m["cpp"][0], cj5 / cpp) < 1e-8
    assert abs(d.average_plaquette(th) - O.average_plaquette(Nt, Nx, th)) < 1e-14
    d.close()


# ---------------------------------------------------------------------------
# Domain wall: independent ensembles, GPU against oracle, within errors
# ---------------------------------------------------------------------------
E_NT, E_NX, E_LS, E_M5, E_MF, E_BETA = 8, 8, 4, 1.0, 0.05, 3.0
E_EPS, E_STEPS, E_NTRAJ, E_CUT, E_THIN, E_BINS = 0.1, 10, 300, 40, 4, 13


def _binned(x, nb):
    n = len(x) // nb * nb
    b = np.asarray(x[:n]).reshape(nb, -1, *np.shape(x)[1:]).mean(1)
    return b.mean(0), b.std(0, ddof=1) / np.sqrt(nb)


def _mres(cpp, cj5):
    """Residual mass: mean over t = 3 .. Nt-4 of <C_J5>/<C_PP>
    (domain_wall/analyze_configs.cpp:98-113)."""
    r = cj5.mean(0) / cpp.mean(0)
    return r[3:cpp.shape[1] - 3].mean()


def _mres_jackknife(cpp, cj5, nb):
    n = len(cpp) // nb * nb
    C = cpp[:n].reshape(nb, -1, cpp.shape[1]).mean(1)
    J = cj5[:n].reshape(nb, -1, cj5.shape[1]).mean(1)
    jk = np.array([_mres(np.delete(C, i, 0), np.delete(J, i, 0)) for i in range(nb)])
    return _mres(C, J), np.sqrt((nb - 1) / nb * ((jk - jk.mean()) ** 2).sum())


def _oracle_ensemble(seed):
    o = O.Dwf(E_NT, E_NX, E_LS, E_M5, E_MF)
    chi, mom, u = O.dwf_draws(seed, E_NTRAJ, o.ndof, o.ngauge)
    th, plaq, kept = np.zeros(o.ngauge), [], []
    for k in range(E_NTRAJ):
        st, prop, inf = o.trajectory(E_BETA, E_EPS, E_STEPS, 1e-10, 5000, th, chi[k], mom[k])
        assert st == 0
        if u[k] < min(np.exp(-inf["dH"]), 1.0):
            th = prop
        plaq.append(O.average_plaquette(E_NT, E_NX, th))
        if k >= E_CUT and (k - E_CUT) % E_THIN == 0:
            kept.append(th.copy())
    cpp, cj5 = [], []
    for c in kept:
        st, a, b = o.cpp_cj5(c, 1e-10, 5000)
        assert st == 0
        cpp.append(a)
        cj5.append(b)
    return np.array(plaq[E_CUT:]), np.array(cpp), np.array(cj5)


def test_independent_ensembles_agree_within_errors(T):
    from three_part_dwf_study_b200.ensemble import hmc_chain

    d = T.DomainWall(E_NT, E_NX, E_LS, E_M5, E_MF, E_BETA)
    cfg, hist = hmc_chain(d, np.zeros(d.Ngauge), E_NTRAJ, seed=11, epsilon=E_EPS, steps=E_STEPS,
                          rtol=1e-10, maxiter=5000, solver=T.SOLVER_MIXED,
                          thermalization_cut=E_CUT, thin=E_THIN)
    m = d.measure(cfg, n_point_times=2, n_wall_times=2, n_noise=0, max_momentum=0, rtol=1e-10,
                  maxiter=5000, solver=T.SOLVER_EO_MIXED)
    d.close()
    g_plaq, g_cpp, g_cj5 = hist["plaquette"][E_CUT:], m["cpp"], m["cj5"]
    o_plaq, o_cpp, o_cj5 = _oracle_ensemble(12)
    assert hist["accepted"].mean() > 0.6
    pairs = {"plaquette": (g_plaq, o_plaq)}
    for t in (1, 2, 4):
        pairs[f"C_PP({t})"] = (g_cpp[:, t], o_cpp[:, t])
    for name, (a, b) in pairs.items():
        ma, ea = _binned(a, E_BINS)
        mb, eb = _binned(b, E_BINS)
        assert abs(ma - mb) < 4 * np.hypot(ea, eb), f"{name}: {ma}+-{ea} vs {mb}+-{eb}"
    ma, ea = _mres_jackknife(g_cpp, g_cj5, E_BINS)
    mb, eb = _mres_jackknife(o_cpp, o_cj5, E_BINS)
    assert abs(ma - mb) < 4 * np.hypot(ea, eb), f"m_res: {ma}+-{ea} vs {mb}+-{eb}"
