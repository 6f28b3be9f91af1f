// Drop-in for domain_wall/include/dwf_operator.hpp: the same entry points,
// computed on the GPU through the C ABI.
#pragma once

#include <cmath>

#include "b200_dwf.hpp"
#include "indexing.hpp"
#include "spin.hpp"

inline Complex link(const Gauge& theta, int mu, int t, int x)
{
    return std::exp(Complex(0.0, theta[gauge_index(mu, t, x)]));
}

inline VectorC b200_dwf_apply(int op, const Gauge& theta, const VectorC& psi)
{
    dwf_ctx* c = b200_dwf_context();
    b200::check(c, dwf_set_gauge(c, 1, theta.data()));
    VectorC out(psi.size());
    b200::check(c, dwf_apply(c, op, 0, b200::cptr(psi), b200::mptr(out), 1));
    return out;
}

inline VectorC apply_D(const Gauge& theta, const VectorC& psi)
{
    return b200_dwf_apply(DWF_OP_D, theta, psi);
}

inline VectorC apply_D_dagger(const Gauge& theta, const VectorC& psi)
{
    return b200_dwf_apply(DWF_OP_DDAG, theta, psi);
}

inline VectorC apply_DD_dagger(const Gauge& theta, const VectorC& psi)
{
    return b200_dwf_apply(DWF_OP_DDDAG, theta, psi);
}

inline VectorC apply_D_dagger_D(const Gauge& theta, const VectorC& psi)
{
    return b200_dwf_apply(DWF_OP_DDAGD, theta, psi);
}
