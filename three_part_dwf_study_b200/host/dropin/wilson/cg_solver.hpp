// Drop-in for wilson/include/cg_solver.hpp: solve_CGNR and solve_DDdag on the
// GPU with the reference's stopping rule, 20*tol guard and messages.
#pragma once

#include "wilson_operator.hpp"

struct SolveResult
{
    VectorC x;
    int iterations;
    double normal_residual;
    double dirac_residual;
};

inline SolveResult solve_CGNR(const WilsonOperator& D, const VectorC& source, double tolerance,
                              int max_iterations)
{
    dwf_ctx* c = b200_wil_context();
    SolveResult r{VectorC(source.size()), 0, 0.0, 0.0};
    double info[3] = {0.0, 0.0, 0.0};
    b200::check(c, wil_solve_cgnr(c, D.theta.data(), b200::cptr(source), tolerance,
                                  max_iterations, b200::solver(), b200::mptr(r.x), info));
    r.iterations = static_cast<int>(info[0]);
    r.normal_residual = info[1];
    r.dirac_residual = info[2];
    return r;
}

inline VectorC solve_DDdag(const WilsonOperator& D, const VectorC& phi, double tolerance,
                           int max_iterations)
{
    dwf_ctx* c = b200_wil_context();
    VectorC eta(phi.size());
    double residual = 0.0;
    b200::check(c, wil_solve_dddag(c, D.theta.data(), b200::cptr(phi), tolerance, max_iterations,
                                   b200::solver(), b200::mptr(eta), &residual));
    return eta;
}
