// Shared helpers of the drop-in headers: status-to-exception mapping and the
// solver path. DWF_B200_SOLVER=cg64 selects the reference FP64 CG everywhere;
// =mixed the full-lattice mixed FP32/FP64 reliable-update CG everywhere;
// otherwise (default) HMC solves use the mixed CG and propagator solves the
// even-odd Schur mixed CG (which ends with the full D^dag D check). All meet
// the same rtol on the FP64 true residual.
#pragma once

#include <complex>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "dwf_b200.h"

namespace b200 {

inline int solver()
{
    static const int s = [] {
        const char* v = std::getenv("DWF_B200_SOLVER");
        return (v && std::strcmp(v, "cg64") == 0) ? DWF_SOLVER_CG64 : DWF_SOLVER_MIXED;
    }();
    return s;
}

// Solver of the propagator (CGNR) solves of the analyzers.
inline int prop_solver()
{
    static const int s = [] {
        const char* v = std::getenv("DWF_B200_SOLVER");
        if (v && std::strcmp(v, "cg64") == 0)
            return int(DWF_SOLVER_CG64);
        if (v && std::strcmp(v, "mixed") == 0)
            return int(DWF_SOLVER_MIXED);
        return int(DWF_SOLVER_EO_MIXED);
    }();
    return s;
}

// CUDA device of this process's contexts: DWF_B200_DEVICE=<n> names one;
// DWF_B200_DEVICE=auto takes the next device in turn among the processes that
// start with it on this host (dwf_round_robin_device on a counter file in
// $TMPDIR or /tmp), so that concurrent study cases spread over the GPUs;
// unset, device 0.
inline int device()
{
    static const int d = [] {
        const char* v = std::getenv("DWF_B200_DEVICE");
        if (!v || !*v)
            return 0;
        if (std::strcmp(v, "auto") != 0)
            return std::atoi(v);
        int n = 0, dev = 0;
        if (dwf_device_count(&n) != DWF_OK || n < 1)
            return 0;
        const char* tmp = std::getenv("TMPDIR");
        const std::string path = std::string(tmp && *tmp ? tmp : "/tmp") + "/dwf_b200_device_counter";
        return dwf_round_robin_device(n, path.c_str(), &dev) == DWF_OK ? dev : 0;
    }();
    return d;
}

inline void check(dwf_ctx* c, int st)
{
    if (st == DWF_OK)
        return;
    const char* m = c ? dwf_last_error(c) : "";
    throw std::runtime_error(m && *m ? std::string(m) : std::string(dwf_status_string(st)));
}

template <typename V>
inline const double* cptr(const V& v)
{
    return reinterpret_cast<const double*>(v.data());
}
template <typename V>
inline double* mptr(V& v)
{
    return reinterpret_cast<double*>(v.data());
}

}  // namespace b200
