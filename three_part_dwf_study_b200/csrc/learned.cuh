// Learned preconditioner: a gauge-equivariant parallel-transport convolution
// (PTC) network N ~ D^-1, trained on the GPU, applied inside a right-
// preconditioned FP32 BiCGStab with FP64 defect correction.
//
// Network: four layers C0 -> H -> H -> H -> C0 (C0 = 2 Ls complex channels per
// 4-D site for domain wall, channel c = 2 s + spin; 2 for Wilson), each
//   out(y)[o] = sum_{k<9} sum_i W_k[o][i] * bf16(T_k(y) * in(y + d_k)[i])
// over the offsets d_k of a 3x3 stencil, T_k the U(1) transporter from y + d_k
// to y (fermion boundary signs included, diagonals the mean of the two
// two-link paths). No bias and no activation: N is linear and gauge
// covariant, and its adjoint is the same chain backwards with
// W'_k = (W_rev(k))^H. Channel mixing runs on the tensor cores (BF16 operands,
// FP32 accumulation).
#pragma once

#include <vector>

#include "context.cuh"

struct LpNet;

namespace dwfb {

constexpr int kLpLayers = 4;

// Release the network and its workspace.
void lp_destroy(dwf_ctx* c);
// Solve D x = src (FP64 device fields) for nrhs sources with the learned
// preconditioner; the stopping rule is the reference's on the normal
// equations, |D^dag (src - D x)| <= rtol |D^dag src|, on the FP64 true residual.
int lp_solve(dwf_ctx* c, int nrhs, const int* conf_h, const double2* src, double2* x,
             double rtol, int maxiter, dwf_solve_info* info);

}  // namespace dwfb
