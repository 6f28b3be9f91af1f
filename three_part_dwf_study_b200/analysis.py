"""Ensemble reductions of the domain-wall analyzer (host side, FP64).

Restates domain_wall/analyze_configs.cpp:78-227 on the per-configuration
outputs of DomainWall.measure():
    averages of C_PP, C_J5                         (:78-96)
    m_res(t) = <C_J5>/<C_PP>, mean over t=3..Nt-4  (:98-113)
    vacuum-subtracted disconnected loop correlator (:115-160)
    eta_singlet = C_pion - eta.flavors * disc      (:151-158)
    momentum-projected pion/disconnected/eta rows  (:177-227)
and writes the reference's CSV files (:172-175, :236-271).
"""
from pathlib import Path

import numpy as np


def residual_mass(cpp_all, cj5_all):
    cpp = np.mean(np.asarray(cpp_all), axis=0)
    cj5 = np.mean(np.asarray(cj5_all), axis=0)
    mres = cj5 / cpp
    Nt = cpp.size
    return cpp, cj5, mres, float(np.mean(mres[3:Nt - 3]))


def disconnected(loops, Nt, Nx):
    """Per-configuration vacuum-subtracted disconnected correlator [nconf, Nt]."""
    L = np.asarray(loops).reshape(-1, Nt, Nx)
    sub = L - L.mean(axis=0, keepdims=True)
    s = sub.sum(axis=2)  # [nconf, Nt]
    out = np.zeros((L.shape[0], Nt))
    for dt in range(Nt):
        out[:, dt] = np.real(np.roll(s, -dt, axis=1) * np.conj(s)).sum(axis=1) / Nt
    return out


def momentum_rows(mom_all, loops, Nt, Nx, flavors):
    """[(n, p, p^2, dt, pion, disconnected, eta)] as the momentum CSV (:177-227)."""
    mom_all = np.asarray(mom_all)
    L = np.asarray(loops).reshape(-1, Nt, Nx)
    nconf = L.shape[0]
    rows = []
    for n in range(mom_all.shape[1]):
        p = 2.0 * np.pi * n / Nx
        lp = (L * np.exp(-1j * p * np.arange(Nx))[None, None, :]).sum(axis=2)
        lpm = lp.mean(axis=0)
        d = lp - lpm
        for dt in range(Nt):
            pion = mom_all[:, n, dt].mean()
            disc = np.real(np.roll(d, -dt, axis=1) * np.conj(d)).sum() / (Nt * nconf)
            rows.append((n, p, p * p, dt, pion, disc, pion - flavors * disc))
    return rows


def reduce_ensemble(meas, Nt, Nx, flavors):
    cpp, cj5, mres, mres_avg = residual_mass(meas["cpp"], meas["cj5"])
    disc_all = disconnected(meas["loop"], Nt, Nx)
    pion_all = np.asarray(meas["mom_cpp"])[:, 0, :]
    eta_all = pion_all - flavors * disc_all
    return dict(cpp=cpp, cj5=cj5, m_res=mres, m_res_average=mres_avg,
                disconnected=disc_all.mean(axis=0), eta=eta_all.mean(axis=0),
                disconnected_all=disc_all, eta_all=eta_all, pion_all=pion_all,
                momentum_rows=momentum_rows(meas["mom_cpp"], meas["loop"], Nt, Nx, flavors))


def _g(v):
    """std::ostream default formatting (6 significant digits)."""
    return f"{v:.6g}"


def write_csvs(red, cpp_all, outdir):
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    Nt = red["cpp"].size
    with open(out / "correlator.csv", "w") as f:
        f.write("t,CPP_average,CJ5_average,m_res,disconnected,eta_singlet\n")
        for t in range(Nt):
            f.write(",".join([str(t), _g(red["cpp"][t]), _g(red["cj5"][t]), _g(red["m_res"][t]),
                              _g(red["disconnected"][t]), _g(red["eta"][t])]) + "\n")
    with open(out / "channels_by_config.csv", "w") as f:
        f.write("config" + "".join(f",pion_t{t}" for t in range(Nt))
                + "".join(f",disconnected_t{t}" for t in range(Nt))
                + "".join(f",eta_t{t}" for t in range(Nt)) + "\n")
        for c in range(len(cpp_all)):
            vals = list(cpp_all[c]) + list(red["disconnected_all"][c]) + list(red["eta_all"][c])
            f.write(str(c) + "".join("," + _g(v) for v in vals) + "\n")
    with open(out / "momentum_correlators.csv", "w") as f:
        f.write("momentum_index,p,p_squared,t,pion,disconnected,eta\n")
        for n, p, p2, dt, pion, disc, eta in red["momentum_rows"]:
            f.write(f"{n},{_g(p)},{_g(p2)},{dt},{_g(pion)},{_g(disc)},{_g(eta)}\n")
