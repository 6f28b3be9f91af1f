// Drop-in for wilson/include/gauge.hpp: actions, forces and hmc_step on the
// GPU. The process-wide random stream and its draw order are the reference's
// (gauge.hpp:16-18, 134-141, 178): momenta, then chi (imaginary part drawn
// first), then the Metropolis uniform.
#pragma once

#include <cmath>
#include <random>
#include <vector>

#include "cg_solver.hpp"

inline std::mt19937_64 rng(random_seed);
inline std::normal_distribution<double> gaussian(0.0, 1.0);
inline std::uniform_real_distribution<double> uniform01(0.0, 1.0);

inline double plaquette_angle(const Gauge& theta, int t, int x)
{
    int tp = (t + 1) % Nt, xp = (x + 1) % Nx;
    return theta[link_index(0, t, x)] + theta[link_index(1, tp, x)] -
           theta[link_index(0, t, xp)] - theta[link_index(1, t, x)];
}

inline double average_plaquette(const Gauge& theta)
{
    dwf_ctx* c = b200_wil_context();
    double p = 0.0;
    b200::check(c, dwf_average_plaquette(c, theta.data(), &p));
    return p;
}

inline double gauge_action_force(const Gauge& theta, Gauge& force)
{
    dwf_ctx* c = b200_wil_context();
    force.assign(ndim * Nt * Nx, 0.0);
    double a = 0.0;
    b200::check(c, dwf_gauge_action_force(c, theta.data(), &a, force.data()));
    return a;
}

inline double pseudofermion_action_force(const Gauge& theta, const VectorC& phi, Gauge& force)
{
    dwf_ctx* c = b200_wil_context();
    force.assign(ndim * Nt * Nx, 0.0);
    double a = 0.0;
    b200::check(c, dwf_pf_action_force(c, theta.data(), b200::cptr(phi), nullptr,
                                       force_cg_tolerance, force_cg_max_iterations,
                                       b200::solver(), &a, force.data(), nullptr, nullptr));
    return a;
}

struct HMCResult
{
    Gauge theta;
    bool accepted;
    double dH;
    double acceptance_probability;
};

inline HMCResult hmc_step(const Gauge& old_theta)
{
    Gauge momentum(ndim * Nt * Nx);
    for (double& p : momentum)
        p = gaussian(rng);
    std::vector<std::complex<double>> chi(Ntot);
    for (int i = 0; i < Ntot; ++i)
    {
        const double im = gaussian(rng);  // the reference's compiler draws this argument first
        const double re = gaussian(rng);
        chi[i] = std::complex<double>(re, im) / std::sqrt(2.0);
    }
    const double u = uniform01(rng);
    dwf_ctx* c = b200_wil_context();
    const dwf_hmc_params hp{hmc_epsilon, hmc_steps, force_cg_tolerance, force_cg_max_iterations,
                            b200::solver()};
    HMCResult r{Gauge(old_theta.size()), false, 0.0, 0.0};
    dwf_traj_info info{};
    b200::check(c, wil_hmc_step(c, &hp, old_theta.data(), momentum.data(),
                                reinterpret_cast<const double*>(chi.data()), u, r.theta.data(),
                                &info));
    r.accepted = info.accepted != 0;
    r.dH = info.dH;
    r.acceptance_probability = info.acceptance_probability;
    return r;
}
