// Golden-vector driver for the domain-wall path (TEST INFRASTRUCTURE).
// Compiled against the UNMODIFIED reference headers (domain_wall/include) and
// the project-written Eigen-API subset in three_part_dwf_study_b200/host/eigen_shim. Reads seeded
// inputs written by tests/golden/make_golden.py from the working directory
// (which also holds the parameters.txt the reference reads at start-up) and
// writes full-precision outputs of the reference entry points:
//   apply_D / apply_D_dagger / apply_DD_dagger / apply_D_dagger_D  (dwf_operator.hpp:15-181)
//   conjugate_gradient                                             (cg_solver.hpp:17-64)
//   pseudofermion_action_force                                     (pseudofermion.hpp:22-166)
//   gauge_action_force, average_plaquette                          (gauge.hpp:26-73)
//   compute_CPP_CJ5, estimate_pseudoscalar_loop_density,
//   compute_momentum_CPP                                           (correlator.hpp:27-310)
#include "correlator.hpp"
#include "gauge.hpp"
#include "npy_io.hpp"
#include "pseudofermion.hpp"

#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

namespace {

VectorC load_field(const std::string& name)
{
    const NpyArray a = load_npy_float64(name);
    if (a.data.size() != static_cast<std::size_t>(2 * Ndof))
        throw std::runtime_error(name + ": wrong size");
    VectorC v(Ndof);
    for (int i = 0; i < Ndof; ++i)
        v[i] = Complex(a.data[2 * i], a.data[2 * i + 1]);
    return v;
}

void save_field(const std::string& name, const VectorC& v)
{
    std::vector<double> d(2 * static_cast<std::size_t>(v.size()));
    for (Eigen::Index i = 0; i < v.size(); ++i)
    {
        d[2 * i] = v[i].real();
        d[2 * i + 1] = v[i].imag();
    }
    save_npy_float64(name, {static_cast<std::size_t>(v.size()), 2}, d);
}

void save_vec(const std::string& name, const std::vector<double>& d)
{
    save_npy_float64(name, {d.size()}, d);
}

}  // namespace

int main()
{
    try
    {
        const NpyArray th = load_npy_float64("in_theta.npy");
        if (th.data.size() != static_cast<std::size_t>(Ngauge))
            throw std::runtime_error("in_theta.npy: wrong size");
        const Gauge theta(th.data.begin(), th.data.end());
        const VectorC psi = load_field("in_psi.npy");
        const VectorC chi = load_field("in_chi.npy");

        save_field("out_D.npy", apply_D(theta, psi));
        save_field("out_Ddag.npy", apply_D_dagger(theta, psi));
        save_field("out_DDdag.npy", apply_DD_dagger(theta, psi));
        save_field("out_DdagD.npy", apply_D_dagger_D(theta, psi));

        // CGNR as the analyzers use it: D^dag D x = D^dag psi.
        const auto normal = [&](const VectorC& v) { return apply_D_dagger_D(theta, v); };
        const VectorC rhs = apply_D_dagger(theta, psi);
        const CgResult cg = conjugate_gradient(normal, rhs, nullptr, propagator_rtol,
                                               propagator_maxiter);
        save_field("out_cg_x.npy", cg.x);
        save_vec("out_cg_info.npy", {double(cg.iterations), cg.relative_residual,
                                     cg.converged ? 1.0 : 0.0});

        // Pseudofermion action and force with phi = D chi (generate_configs.cpp:64).
        const VectorC phi = apply_D(theta, chi);
        const PseudofermionActionForce pf = pseudofermion_action_force(theta, phi, nullptr);
        save_vec("out_pf_force.npy", pf.force);
        save_field("out_pf_eta.npy", pf.eta);
        save_vec("out_pf_info.npy", {pf.action, double(pf.iterations), pf.relative_residual});

        // Warm-started solve, as in the leapfrog steps (generate_configs.cpp:119-126).
        const PseudofermionActionForce pf2 = pseudofermion_action_force(theta, phi, &pf.eta);
        save_vec("out_pf_warm_info.npy",
                 {pf2.action, double(pf2.iterations), pf2.relative_residual});

        const GaugeActionForce g = gauge_action_force(theta);
        save_vec("out_gauge_force.npy", g.force);
        save_vec("out_gauge_info.npy", {g.action, average_plaquette(theta)});

        const CorrelatorPair cc = compute_CPP_CJ5(theta);
        save_vec("out_cpp.npy", cc.CPP);
        save_vec("out_cj5.npy", cc.CJ5);

        const ComplexCorr loop = estimate_pseudoscalar_loop_density(theta, eta_random_seed);
        std::vector<double> ld(2 * loop.size());
        for (std::size_t i = 0; i < loop.size(); ++i)
        {
            ld[2 * i] = loop[i].real();
            ld[2 * i + 1] = loop[i].imag();
        }
        save_npy_float64("out_loop.npy", {loop.size(), 2}, ld);

        const std::vector<Corr> mom = compute_momentum_CPP(theta);
        std::vector<double> md;
        for (const Corr& c : mom)
            md.insert(md.end(), c.begin(), c.end());
        save_npy_float64("out_mom.npy", {mom.size(), static_cast<std::size_t>(Nt)}, md);
        return 0;
    }
    catch (const std::exception& e)
    {
        std::cerr << "error: " << e.what() << '\n';
        return 1;
    }
}
