// Drop-in for domain_wall/include/cg_solver.hpp.
//
// Two forms of conjugate_gradient:
//  * conjugate_gradient(op, theta, b, guess, rtol, maxiter) names the normal
//    operator (DWF_OP_DDDAG or DWF_OP_DDAGD on a gauge field) and runs the
//    whole solve on the GPU (dwf_cg). The drop-in headers' own callers
//    (pseudofermion.hpp, correlator.hpp) use this form.
//  * conjugate_gradient(apply_A, b, guess, rtol, maxiter) keeps the reference's
//    signature (domain_wall/include/cg_solver.hpp:17-22) for callers that pass
//    the operator as a std::function. When apply_A holds a b200::NormalOperator
//    the call is the GPU solve above. Any other callable is the caller's own
//    host code, which the GPU cannot run: the CG recurrences then run on the
//    host around it (the callable may itself call the GPU operators, e.g.
//    apply_D_dagger_D), with the reference's rules.
// Both return the reference's CgResult.
#pragma once

#include <cmath>
#include <functional>
#include <stdexcept>

#include "b200_dwf.hpp"
#include "dwf_operator.hpp"

struct CgResult
{
    VectorC x;
    int iterations;
    double relative_residual;
    bool converged;
};

namespace b200 {

// A normal operator of the domain-wall context, known to the GPU solver by
// name: b200::NormalOperator{DWF_OP_DDAGD, theta} wrapped in the std::function
// that conjugate_gradient takes solves on the GPU.
struct NormalOperator
{
    int op;  // DWF_OP_DDDAG or DWF_OP_DDAGD
    Gauge theta;
    VectorC operator()(const VectorC& v) const { return b200_dwf_apply(op, theta, v); }
};

}  // namespace b200

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

inline CgResult conjugate_gradient(const std::function<VectorC(const VectorC&)>& apply_A,
                                   const VectorC& b, const VectorC* initial_guess, double rtol,
                                   int maxiter)
{
    if (const b200::NormalOperator* n = apply_A.target<b200::NormalOperator>())
        return conjugate_gradient(n->op, n->theta, b, initial_guess, rtol, maxiter);
    // Host recurrences around the caller's operator. Same contract as the
    // reference: x0 = guess or 0; a zero right-hand side returns x0 at once;
    // stop when the recursive residual |r| <= rtol |b|; a vanishing <p, A p>
    // throws.
    VectorC x = initial_guess ? *initial_guess : VectorC::Zero(b.size());
    VectorC r = b - apply_A(x);
    const double bnorm = b.norm();
    if (bnorm == 0.0)
        return {x, 0, 0.0, true};
    double rr = std::real(r.dot(r));
    double rel = std::sqrt(rr) / bnorm;
    if (rel <= rtol)
        return {x, 0, rel, true};
    VectorC p = r;
    for (int k = 1; k <= maxiter; ++k)
    {
        const VectorC q = apply_A(p);
        const Complex pq = p.dot(q);
        if (std::abs(pq) == 0.0)
            throw std::runtime_error("CG encountered a zero denominator");
        const double a = rr / std::real(pq);
        x += a * p;
        r -= a * q;
        const double rr_next = std::real(r.dot(r));
        rel = std::sqrt(rr_next) / bnorm;
        if (rel <= rtol)
            return {x, k, rel, true};
        p = r + (rr_next / rr) * p;
        rr = rr_next;
    }
    return {x, maxiter, rel, false};
}
