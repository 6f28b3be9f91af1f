// Per-thread Wilson context built from the parameters the reference reads at
// start-up (wilson/include/parameters.hpp:6-44).
#pragma once

#include "../b200_common.hpp"
#include "parameters.hpp"
#include "types.hpp"

inline dwf_ctx* b200_wil_context()
{
    thread_local struct Holder
    {
        dwf_ctx* c = nullptr;
        Holder()
        {
            const wil_params p{Nt, Nx, m0, beta, time_boundary_sign, space_boundary_sign, b200::device()};
            b200::check(nullptr, wil_ctx_create(&p, &c));
        }
        ~Holder() { dwf_ctx_destroy(c); }
    } holder;
    return holder.c;
}
