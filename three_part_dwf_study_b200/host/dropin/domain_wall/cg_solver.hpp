// Drop-in for domain_wall/include/cg_solver.hpp. The reference's solver takes
// the operator as a std::function; on the GPU the operator is named instead
// (DWF_OP_DDDAG or DWF_OP_DDAGD on a gauge field), and the result type is the
// reference's CgResult.
#pragma once

#include "b200_dwf.hpp"

struct CgResult
{
    VectorC x;
    int iterations;
    double relative_residual;
    bool converged;
};

inline CgResult conjugate_gradient(int op, const Gauge& theta, const VectorC& b,
                                   const VectorC* initial_guess, double rtol, int maxiter)
{
    dwf_ctx* c = b200_dwf_context();
    b200::check(c, dwf_set_gauge(c, 1, theta.data()));
    VectorC x = initial_guess ? *initial_guess : VectorC::Zero(b.size());
    dwf_solve_info info{};
    const int st = dwf_cg(c, op, 0, b200::cptr(b), b200::mptr(x), initial_guess != nullptr,
                          rtol, maxiter, b200::solver(), &info);
    if (st == DWF_ZERO_DENOM)
        throw std::runtime_error("CG encountered a zero denominator");
    if (st != DWF_OK && st != DWF_NOT_CONVERGED)
        b200::check(c, st);
    return {x, info.iterations, info.relres, info.converged != 0};
}
