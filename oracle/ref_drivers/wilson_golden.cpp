// Golden-vector driver for the Wilson path (TEST INFRASTRUCTURE).
// Compiled against the UNMODIFIED reference headers (wilson/include, plus the
// .npy reader/writer from domain_wall/include/npy_io.hpp) and the project-written
// Eigen-API subset in three_part_dwf_study_b200/host/eigen_shim. Writes full-precision outputs of:
//   build_wilson_matrix (wilson_operator.hpp:10-62) applied as D psi and D^dag psi
//   solve_CGNR, solve_DDdag (cg_solver.hpp:19-78)
//   gauge_action_force, pseudofermion_action_force, average_plaquette (gauge.hpp:20-122)
//   hmc_step x3 from a hot start, with the reference's global RNG (gauge.hpp:16-18,124-180)
//   pseudoscalar_correlator (correlator.hpp:10-40)
#include "correlator.hpp"
#include "gauge.hpp"
#include "npy_io.hpp"

#include <iostream>
#include <string>
#include <vector>

namespace {

VectorC load_field(const std::string& name)
{
    const NpyArray a = load_npy_float64(name);
    if (a.data.size() != static_cast<std::size_t>(2 * Ntot))
        throw std::runtime_error(name + ": wrong size");
    VectorC v(Ntot);
    for (int i = 0; i < Ntot; ++i)
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
        if (th.data.size() != static_cast<std::size_t>(ndim * Nt * Nx))
            throw std::runtime_error("in_theta.npy: wrong size");
        const Gauge theta(th.data.begin(), th.data.end());
        const VectorC psi = load_field("in_psi.npy");

        const SparseC D = build_wilson_matrix(theta);
        save_field("out_D.npy", D * psi);
        save_field("out_Ddag.npy", D.adjoint() * psi);

        const SolveResult s = solve_CGNR(D, psi, measurement_cg_tolerance,
                                         measurement_cg_max_iterations);
        save_field("out_cgnr_x.npy", s.x);
        save_vec("out_cgnr_info.npy",
                 {double(s.iterations), s.normal_residual, s.dirac_residual});

        const VectorC eta = solve_DDdag(D, psi, force_cg_tolerance, force_cg_max_iterations);
        save_field("out_dddag_x.npy", eta);

        Gauge fg;
        const double sg = gauge_action_force(theta, fg);
        save_vec("out_gauge_force.npy", fg);
        Gauge fpf;
        const double spf = pseudofermion_action_force(theta, psi, fpf);
        save_vec("out_pf_force.npy", fpf);
        save_vec("out_actions.npy", {sg, spf, average_plaquette(theta)});

        save_vec("out_corr.npy", pseudoscalar_correlator(theta));

        // Three HMC steps from the input configuration, drawing from the
        // reference's process-wide mt19937_64(wilson.random_seed).
        std::vector<double> thetas;
        std::vector<double> info;
        Gauge current = theta;
        for (int k = 0; k < 3; ++k)
        {
            const HMCResult r = hmc_step(current);
            current = r.theta;
            thetas.insert(thetas.end(), current.begin(), current.end());
            info.push_back(r.dH);
            info.push_back(r.acceptance_probability);
            info.push_back(r.accepted ? 1.0 : 0.0);
        }
        save_npy_float64("out_hmc_theta.npy",
                         {3, 2, static_cast<std::size_t>(Nt), static_cast<std::size_t>(Nx)},
                         thetas);
        save_npy_float64("out_hmc_info.npy", {3, 3}, info);
        return 0;
    }
    catch (const std::exception& e)
    {
        std::cerr << "error: " << e.what() << '\n';
        return 1;
    }
}
