// Drop-in for wilson/include/wilson_operator.hpp. The reference assembles D as
// an Eigen sparse matrix on every call; here build_wilson_matrix returns a
// matrix-free handle whose products (D * v, D.adjoint() * v) run on the GPU.
#pragma once

#include "b200_wil.hpp"
#include "indexing.hpp"

struct WilsonOperator
{
    Gauge theta;
    bool dagger = false;
    WilsonOperator adjoint() const { return {theta, !dagger}; }
};

inline WilsonOperator build_wilson_matrix(const Gauge& theta) { return {theta, false}; }

inline VectorC operator*(const WilsonOperator& D, const VectorC& v)
{
    dwf_ctx* c = b200_wil_context();
    b200::check(c, dwf_set_gauge(c, 1, D.theta.data()));
    VectorC out(v.size());
    b200::check(c, dwf_apply(c, D.dagger ? DWF_OP_DDAG : DWF_OP_D, 0, b200::cptr(v),
                             b200::mptr(out), 1));
    return out;
}
