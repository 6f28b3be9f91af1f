// Drop-in for wilson/include/correlator.hpp: both point-source solves and the
// contraction C(t) = sum_{x,a,b} |S(t,x,a;b)|^2 on the GPU.
#pragma once

#include <iostream>

#include "b200_wil.hpp"

inline Corr pseudoscalar_correlator(const Gauge& theta)
{
    dwf_ctx* c = b200_wil_context();
    Corr C(Nt, 0.0);
    dwf_solve_info info[2];
    b200::check(c, wil_pseudoscalar_correlator(c, 1, theta.data(), source_t, source_x,
                                               measurement_cg_tolerance,
                                               measurement_cg_max_iterations, b200::solver(),
                                               C.data(), info));
    for (int b = 0; b < Ns; ++b)
        std::cout << "    spin=" << b << " CG iterations=" << info[b].iterations
                  << " normal residual=" << info[b].true_relres
                  << " D residual=" << info[b].dirac_relres << "\n";
    return C;
}
