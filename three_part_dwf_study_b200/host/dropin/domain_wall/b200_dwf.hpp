// Per-thread domain-wall context built from the parameters the reference
// reads at start-up (domain_wall/include/parameters.hpp:7-41).
#pragma once

#include "../b200_common.hpp"
#include "parameters.hpp"
#include "types.hpp"

inline dwf_ctx* b200_dwf_context()
{
    thread_local struct Holder
    {
        dwf_ctx* c = nullptr;
        Holder()
        {
            const dwf_params p{Nt, Nx, N5, M5, mf, beta, b200::device()};
            b200::check(nullptr, dwf_ctx_create(&p, &c));
        }
        ~Holder() { dwf_ctx_destroy(c); }
    } holder;
    return holder.c;
}
