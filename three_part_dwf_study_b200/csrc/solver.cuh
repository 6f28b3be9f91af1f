// Persistent multi-right-hand-side CG kernels.
#pragma once

#include "dirac.cuh"

namespace dwfb {

// Per-right-hand-side state codes held in shared memory during a solve.
enum : int
{
    RHS_ACTIVE = -1,
};

struct SolveDesc
{
    Lat L;
    int dag_first;  // 1: A = D D^dag (D^dag applied first); 0: A = D^dag D
    int nrhs;
    long fsz;       // complex elements per right-hand-side field (2 * nsite)
    const int* rhs_conf;  // device [nrhs] configuration index per right-hand side
    const double2* U64;   // [nconf][2V]
    const float2* U32;
    long usz;             // link elements per configuration (2V)
    const double2* b;
    double2* x;
    double2* r;
    double2* p;    // search direction, double-buffered with p2
    double2* p2;
    double2* t;
    float2* r32;
    float2* p32;   // FP32 search direction, double-buffered with p32b
    float2* p32b;
    float2* t32;
    float2* e32;
    double* part;  // partial sums [nrhs][nch][2]
    int nch, ch;   // chunks per right-hand side and sites per chunk
    double rtol;
    int maxiter;
    int has_guess;
    const int* active_in;  // device [nrhs] or null: right-hand sides with 0 are left untouched
    int eigen_rule;   // stop at |r|^2 < tol^2 |b|^2 and count as Eigen's ConjugateGradient
    double delta;     // reliable-update trigger: |r32| < delta * |r| at the last update
    int stall_limit;  // consecutive non-improving reliable updates before giving up
    // reliable updates run only at iterations divisible by ru_period (and at
    // maxiter), so that the right-hand sides of a batch that want one share the
    // FP64 phases instead of each paying them at its own iteration (0 or 1:
    // every iteration)
    int ru_period;
    // outputs (device, [nrhs])
    int* out_iters;
    double* out_relres;
    int* out_status;
    int* out_ru;
    GridBar* bar;
    unsigned long long timeout_ns;
    unsigned expected_blocks;  // normally gridDim.x
};

// Reliable-update period of the mixed solvers (iterations).
#ifndef DWFB_RU_PERIOD
#define DWFB_RU_PERIOD 16
#endif
constexpr int kRuPeriod = DWFB_RU_PERIOD;

// Dynamic shared memory needed by the solver kernels for nrhs right-hand sides.
__host__ __device__ inline size_t solver_smem_bytes(int nrhs)
{
    return 64 * sizeof(double) + size_t(nrhs) * (6 * sizeof(double) + 5 * sizeof(int));
}

template <bool FUSED, int MINB>
__global__ void cg64_kernel(SolveDesc d);
template <bool FUSED, int MINB>
__global__ void cg_mixed_kernel(SolveDesc d);

}  // namespace dwfb
