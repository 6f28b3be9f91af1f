// CPU timing driver for the reference's domain-wall propagator solve
// (TEST/BENCH INFRASTRUCTURE). Compiled against the UNMODIFIED reference
// headers and the Eigen-API subset in oracle/eigen_shim.
//
// Usage (in a directory holding parameters.txt and in_theta.npy):
//   ref_bench <nsolves> [threads]
// Solves D^dag D x = D^dag src for `nsolves` boundary point sources exactly as
// compute_momentum_CPP builds them (domain_wall/include/correlator.hpp:129-146):
// source spin b = i % 2, source time t_src = ((i / 2) % 4) * Nt / 4, x = 0, with
// conjugate_gradient(apply_D_dagger_D, ...) (cg_solver.hpp:17-64) at
// dwf.propagator_rtol / dwf.propagator_maxiter. Independent solves run on
// OpenMP threads, one solve per thread at a time, which is how the reference's
// analyzer spreads work (domain_wall/analyze_configs.cpp:45).
// Prints one JSON line with the wall time and per-solve iteration counts.
#include "cg_solver.hpp"
#include "dwf_operator.hpp"
#include "npy_io.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <omp.h>
#include <vector>

int main(int argc, char** argv)
{
    try
    {
        const int nsolves = argc > 1 ? std::atoi(argv[1]) : 1;
        if (argc > 2)
            omp_set_num_threads(std::atoi(argv[2]));
        const NpyArray th = load_npy_float64("in_theta.npy");
        if (th.data.size() != static_cast<std::size_t>(Ngauge))
            throw std::runtime_error("in_theta.npy: wrong size");
        const Gauge theta(th.data.begin(), th.data.end());
        const Eigen::Matrix2cd PL = projector_L();
        const Eigen::Matrix2cd PR = projector_R();

        std::vector<int> iters(nsolves, 0);
        std::vector<double> relres(nsolves, 0.0);
        std::vector<int> conv(nsolves, 0);
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic)
        for (int i = 0; i < nsolves; ++i)
        {
            const int b = i % 2;
            const int t_src = ((i / 2) % 4) * Nt / 4;
            VectorC source = VectorC::Zero(Ndof);
            for (int spin = 0; spin < Ns; ++spin)
            {
                source[fermion_index(0, t_src, 0, spin)] += PL(spin, b);
                source[fermion_index(N5 - 1, t_src, 0, spin)] += PR(spin, b);
            }
            const VectorC rhs = apply_D_dagger(theta, source);
            const auto apply_M = [&](const VectorC& v) { return apply_D_dagger_D(theta, v); };
            const CgResult r = conjugate_gradient(apply_M, rhs, nullptr, propagator_rtol,
                                                  propagator_maxiter);
            iters[i] = r.iterations;
            relres[i] = r.relative_residual;
            conv[i] = r.converged ? 1 : 0;
        }
        const auto t1 = std::chrono::steady_clock::now();
        const double secs = std::chrono::duration<double>(t1 - t0).count();
        std::printf("{\"seconds\": %.9g, \"solves\": %d, \"threads\": %d, \"iterations\": [",
                    secs, nsolves, omp_get_max_threads());
        for (int i = 0; i < nsolves; ++i)
            std::printf("%s%d", i ? ", " : "", iters[i]);
        std::printf("], \"relres\": [");
        for (int i = 0; i < nsolves; ++i)
            std::printf("%s%.6e", i ? ", " : "", relres[i]);
        std::printf("], \"converged\": [");
        for (int i = 0; i < nsolves; ++i)
            std::printf("%s%d", i ? ", " : "", conv[i]);
        std::printf("]}\n");
        return 0;
    }
    catch (const std::exception& e)
    {
        std::cerr << "error: " << e.what() << '\n';
        return 1;
    }
}
