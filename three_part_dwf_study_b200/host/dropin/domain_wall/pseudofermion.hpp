// Drop-in for domain_wall/include/pseudofermion.hpp: eta = (D D^dag)^-1 phi
// (warm-started from eta_guess), S = Re<phi, eta> and its force, on the GPU.
#pragma once

#include "b200_dwf.hpp"

struct PseudofermionActionForce
{
    double action;
    Gauge force;
    VectorC eta;
    int iterations;
    double relative_residual;
};

inline PseudofermionActionForce pseudofermion_action_force(const Gauge& theta, const VectorC& phi,
                                                           const VectorC* eta_guess)
{
    dwf_ctx* c = b200_dwf_context();
    PseudofermionActionForce r{0.0, Gauge(Ngauge, 0.0), VectorC(Ndof), 0, 0.0};
    dwf_solve_info info{};
    const int st = dwf_pf_action_force(c, theta.data(), b200::cptr(phi),
                                       eta_guess ? b200::cptr(*eta_guess) : nullptr,
                                       pseudofermion_rtol, pseudofermion_maxiter, b200::solver(),
                                       &r.action, r.force.data(), b200::mptr(r.eta), &info);
    b200::check(c, st);  // "Pseudofermion CG failed to converge"
    r.iterations = info.iterations;
    r.relative_residual = info.relres;
    return r;
}
