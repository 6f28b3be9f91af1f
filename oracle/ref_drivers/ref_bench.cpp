// CPU timing driver for the reference's domain-wall hot path
// (TEST/BENCH INFRASTRUCTURE). Compiled against the UNMODIFIED reference
// headers and the Eigen-API subset in three_part_dwf_study_b200/host/eigen_shim.
// Runs in a directory holding parameters.txt and in_theta.npy.
//
//   ref_bench solve <threads> <first> <count>
//       Complete propagator solves of sources first .. first+count-1 (taken
//       modulo their number) of in_src.npy ([n][Ndof][2] float64, complex
//       sources in the fermion_index layout), each exactly as the reference's
//       analyzer solves a source (domain_wall/include/correlator.hpp:77-79,
//       :139-142, :213-220): rhs = apply_D_dagger(theta, source), then
//       conjugate_gradient(apply_D_dagger_D, rhs, nullptr, dwf.propagator_rtol,
//       dwf.propagator_maxiter) (cg_solver.hpp:17-64). Independent solves run
//       on OpenMP threads, one solve per thread at a time, which is how the
//       reference's analyzer spreads work (domain_wall/analyze_configs.cpp:45).
//   ref_bench apply <reps>
//       apply_D (dwf_operator.hpp:15-92) on a seeded Gaussian field, `reps`
//       back-to-back calls on one thread (the reference's operator is serial).
//
// Prints one JSON line: wall seconds and, for solves, per-solve iterations,
// relative residuals and convergence flags.
#include "cg_solver.hpp"
#include "dwf_operator.hpp"
#include "npy_io.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <omp.h>
#include <random>
#include <vector>

namespace {

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int run_solves(const Gauge& theta, int threads, int first, int count)
{
    const NpyArray src = load_npy_float64("in_src.npy");
    const std::size_t per = static_cast<std::size_t>(Ndof) * 2;
    if (src.data.size() % per != 0 || src.data.empty())
        throw std::runtime_error("in_src.npy: wrong size");
    const int nsrc = static_cast<int>(src.data.size() / per);
    omp_set_num_threads(threads);
    std::vector<int> iters(count, 0);
    std::vector<double> relres(count, 0.0);
    std::vector<int> conv(count, 0);
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < count; ++i)
    {
        const int k = (first + i) % nsrc;
        VectorC source(Ndof);
        for (int j = 0; j < Ndof; ++j)
            source[j] = Complex(src.data[k * per + 2 * j], src.data[k * per + 2 * j + 1]);
        const VectorC rhs = apply_D_dagger(theta, source);
        const auto apply_M = [&](const VectorC& v) { return apply_D_dagger_D(theta, v); };
        const CgResult r = conjugate_gradient(apply_M, rhs, nullptr, propagator_rtol,
                                              propagator_maxiter);
        iters[i] = r.iterations;
        relres[i] = r.relative_residual;
        conv[i] = r.converged ? 1 : 0;
    }
    const double secs = seconds_since(t0);
    std::printf("{\"seconds\": %.9g, \"solves\": %d, \"threads\": %d, \"iterations\": [",
                secs, count, threads);
    for (int i = 0; i < count; ++i)
        std::printf("%s%d", i ? ", " : "", iters[i]);
    std::printf("], \"relres\": [");
    for (int i = 0; i < count; ++i)
        std::printf("%s%.6e", i ? ", " : "", relres[i]);
    std::printf("], \"converged\": [");
    for (int i = 0; i < count; ++i)
        std::printf("%s%d", i ? ", " : "", conv[i]);
    std::printf("]}\n");
    return 0;
}

int run_apply(const Gauge& theta, int reps)
{
    std::mt19937_64 rng(7);
    std::normal_distribution<double> normal(0.0, 1.0);
    VectorC psi(Ndof);
    for (int i = 0; i < Ndof; ++i)
        psi[i] = Complex(normal(rng), normal(rng));
    VectorC out = apply_D(theta, psi);  // warm-up
    const auto t0 = std::chrono::steady_clock::now();
    double sink = 0.0;
    for (int r = 0; r < reps; ++r)
    {
        out = apply_D(theta, psi);
        sink += std::real(out[r % Ndof]);
    }
    const double secs = seconds_since(t0);
    std::printf("{\"seconds\": %.9g, \"reps\": %d, \"threads\": 1, \"checksum\": %.6e}\n", secs,
                reps, sink);
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    try
    {
        if (argc < 2)
            throw std::runtime_error("usage: ref_bench solve <threads> <first> <count> | apply <reps>");
        const NpyArray th = load_npy_float64("in_theta.npy");
        if (th.data.size() != static_cast<std::size_t>(Ngauge))
            throw std::runtime_error("in_theta.npy: wrong size");
        const Gauge theta(th.data.begin(), th.data.end());
        if (std::strcmp(argv[1], "solve") == 0 && argc == 5)
            return run_solves(theta, std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]));
        if (std::strcmp(argv[1], "apply") == 0 && argc == 3)
            return run_apply(theta, std::atoi(argv[2]));
        throw std::runtime_error("usage: ref_bench solve <threads> <first> <count> | apply <reps>");
    }
    catch (const std::exception& e)
    {
        std::cerr << "error: " << e.what() << '\n';
        return 1;
    }
}
