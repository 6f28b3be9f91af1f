// Drop-in for domain_wall/include/correlator.hpp: the boundary wall, point and
// Z4-noise propagators and their contractions, solved and contracted on the
// GPU (one batched solve per call).
#pragma once

#include <array>
#include <complex>
#include <iostream>
#include <stdexcept>
#include <utility>
#include <vector>

#include "b200_dwf.hpp"
#include "indexing.hpp"
#include "spin.hpp"

struct CorrelatorPair
{
    Corr CPP;
    Corr CJ5;
};

using ComplexCorr = std::vector<Complex>;

inline ComplexCorr estimate_pseudoscalar_loop_density(const Gauge& theta, unsigned long long seed)
{
    if (eta_noise_vectors < 1)
        throw std::runtime_error("eta.noise_vectors must be positive");
    dwf_ctx* c = b200_dwf_context();
    // the reference's stream: mt19937_64(seed), digits drawn noise, t, x, spin
    std::vector<signed char> z4(static_cast<std::size_t>(eta_noise_vectors) * Nt * Nx * Ns);
    b200::check(c, dwf_z4_digits(seed, static_cast<long>(z4.size()), z4.data()));
    const dwf_measure_params mp{0, 0, eta_noise_vectors, 0, propagator_rtol, propagator_maxiter,
                                b200::prop_solver()};
    ComplexCorr loop(static_cast<std::size_t>(Nt) * Nx);
    std::vector<dwf_solve_info> info(eta_noise_vectors);
    b200::check(c, dwf_measure(c, &mp, 1, theta.data(), z4.data(), nullptr, nullptr,
                               reinterpret_cast<double*>(loop.data()), nullptr, info.data()));
    for (const dwf_solve_info& i : info)
        if (!i.converged)
            throw std::runtime_error("Eta loop CGNR failed to converge");
    return loop;
}

inline std::vector<Corr> compute_momentum_CPP(const Gauge& theta)
{
    if (max_momentum < 0 || max_momentum > Nx / 2)
        throw std::runtime_error("analysis.max_momentum is outside 0..Nx/2");
    dwf_ctx* c = b200_dwf_context();
    const dwf_measure_params mp{2, 0, 0, max_momentum, propagator_rtol, propagator_maxiter,
                                b200::prop_solver()};
    std::vector<double> mom(static_cast<std::size_t>(max_momentum + 1) * Nt);
    std::vector<dwf_solve_info> info(4);
    b200::check(c, dwf_measure(c, &mp, 1, theta.data(), nullptr, nullptr, nullptr, nullptr,
                               mom.data(), info.data()));
    for (const dwf_solve_info& i : info)
        if (!i.converged)
            throw std::runtime_error("Momentum propagator CGNR failed to converge");
    std::vector<Corr> result(max_momentum + 1, Corr(Nt, 0.0));
    for (int n = 0; n <= max_momentum; ++n)
        for (int t = 0; t < Nt; ++t)
            result[n][t] = mom[static_cast<std::size_t>(n) * Nt + t];
    return result;
}

inline void b200_print_wall_solve(int t_src, int spin, const dwf_solve_info& i)
{
    if (!i.converged)
        std::cout << "    CGNR info = nonzero\n";
    std::cout << "    t_src=" << t_src << " spin=" << spin << " iterations=" << i.iterations
              << " normal residual=" << i.relres << " D residual=" << i.dirac_relres << '\n';
}

inline std::array<VectorC, 2> boundary_wall_source_propagator(const Gauge& theta, int t_src)
{
    dwf_ctx* c = b200_dwf_context();
    b200::check(c, dwf_set_gauge(c, 1, theta.data()));
    const Eigen::Matrix2cd PL = projector_L();
    const Eigen::Matrix2cd PR = projector_R();
    std::vector<Complex> src(2 * static_cast<std::size_t>(Ndof), Complex(0.0, 0.0));
    for (int b = 0; b < Ns; ++b)
        for (int x = 0; x < Nx; ++x)
            for (int spin = 0; spin < Ns; ++spin)
            {
                src[static_cast<std::size_t>(b) * Ndof + fermion_index(0, t_src, x, spin)] +=
                    PL(spin, b);
                src[static_cast<std::size_t>(b) * Ndof + fermion_index(N5 - 1, t_src, x, spin)] +=
                    PR(spin, b);
            }
    std::vector<Complex> x(src.size());
    dwf_solve_info info[2];
    b200::check(c, dwf_propagators(c, 2, nullptr, reinterpret_cast<const double*>(src.data()),
                                   reinterpret_cast<double*>(x.data()), propagator_rtol,
                                   propagator_maxiter, b200::prop_solver(), info));
    std::array<VectorC, 2> props;
    for (int b = 0; b < Ns; ++b)
    {
        b200_print_wall_solve(t_src, b, info[b]);
        props[b] = VectorC(Ndof);
        for (int i = 0; i < Ndof; ++i)
            props[b][i] = x[static_cast<std::size_t>(b) * Ndof + i];
    }
    return props;
}

inline CorrelatorPair compute_CPP_CJ5(const Gauge& theta)
{
    dwf_ctx* c = b200_dwf_context();
    const dwf_measure_params mp{0, 2, 0, 0, propagator_rtol, propagator_maxiter, b200::prop_solver()};
    CorrelatorPair out{Corr(Nt, 0.0), Corr(Nt, 0.0)};
    dwf_solve_info info[4];
    b200::check(c, dwf_measure(c, &mp, 1, theta.data(), nullptr, out.CPP.data(), out.CJ5.data(),
                               nullptr, nullptr, info));
    for (int k = 0; k < 4; ++k)
        b200_print_wall_solve((k / 2) * Nt / 2, k % 2, info[k]);
    return out;
}
