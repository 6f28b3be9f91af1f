// HMC kernels: gauge action/force, pseudofermion force, momentum kick and
// link drift, and deterministic FP64 reductions.
#pragma once

#include "common.cuh"

namespace dwfb {

constexpr int kRedBlocks = 64;  // blocks of the partial-sum kernels

// Gauge force F = dS_g/dtheta and per-block partials of S_g = beta sum (1 - cos P)
// and sum cos P (domain_wall/include/gauge.hpp:15-73, wilson/include/gauge.hpp:20-62).
__global__ void gauge_force_kernel(int Nt, int Nx, double beta, const double* __restrict__ th,
                                   double* __restrict__ force, double* __restrict__ part);

// force[l] += pseudofermion force on link l from eta and xi = D^dag eta
// (domain_wall/include/pseudofermion.hpp:45-157, wilson/include/gauge.hpp:75-119).
__global__ void pf_force_kernel(Lat L, const double2* __restrict__ eta,
                                const double2* __restrict__ xi, const double2* __restrict__ U,
                                double* __restrict__ force);

// part[b] = partial sums of Re(a^dag b) over n complex entries.
__global__ void dot_re_kernel(const double2* __restrict__ a, const double2* __restrict__ b, long n,
                              double* __restrict__ part);
// part[b] = partial sums of 0.5 * p^2.
__global__ void kinetic_kernel(const double* __restrict__ p, long n, double* __restrict__ part);
// out[slot] = sum of part[0..nblk) with stride `stride`, fixed order (one block).
__global__ void finish_sum_kernel(const double* __restrict__ part, int nblk, int stride,
                                  double* __restrict__ out);
// mom -= c * force
__global__ void kick_kernel(double* __restrict__ mom, const double* __restrict__ force, double c,
                            long n);
// theta += eps * mom (wrapped into [-pi, pi) when `wrap`), links recomputed.
__global__ void drift_kernel(double* __restrict__ th, const double* __restrict__ mom, double eps,
                             int wrap, long n, double2* __restrict__ U64, float2* __restrict__ U32);

}  // namespace dwfb
