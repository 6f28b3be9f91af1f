// C ABI: gauge/pseudofermion action and force, HMC trajectories (domain wall
// and Wilson), and the Wilson context and solver entry points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "context.cuh"
#include "hmc.cuh"
#include "kernels.cuh"

using namespace dwfb;

#define CK(call)                                                                        \
    do                                                                                  \
    {                                                                                   \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ctx_fail(c, DWF_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

namespace {

int ensure_hmc(dwf_ctx* c)
{
    if (c->h_mom)
        return DWF_OK;
    const size_t ng = size_t(c->usz());
    const size_t f = size_t(c->fsz());
    CK(cudaMalloc(&c->h_mom, ng * sizeof(double)));
    CK(cudaMalloc(&c->h_force, ng * sizeof(double)));
    CK(cudaMalloc(&c->h_part, 2 * kRedBlocks * sizeof(double)));
    CK(cudaMalloc(&c->h_scal, 16 * sizeof(double)));
    CK(cudaMalloc(&c->h_chi, f * sizeof(double2)));
    CK(cudaMalloc(&c->h_phi, f * sizeof(double2)));
    CK(cudaMalloc(&c->h_eta, f * sizeof(double2)));
    CK(cudaMalloc(&c->h_xi, f * sizeof(double2)));
    CK(cudaMemset(c->h_eta, 0, f * sizeof(double2)));
    return DWF_OK;
}

// Gauge force of configuration slot 0 into h_force; S_g and sum cos P to host.
int gauge_force(dwf_ctx* c, double* Sg, double* cos_sum)
{
    gauge_force_kernel<<<kRedBlocks, 256, 0, c->stream>>>(c->L.Nt, c->L.Nx, c->beta, c->theta,
                                                          c->h_force, c->h_part);
    finish_sum_kernel<<<1, 64, 0, c->stream>>>(c->h_part, kRedBlocks, 2, c->h_scal + 0);
    finish_sum_kernel<<<1, 64, 0, c->stream>>>(c->h_part + 1, kRedBlocks, 2, c->h_scal + 1);
    CK(cudaGetLastError());
    c->launches += 3;
    double h[2];
    CK(cudaMemcpyAsync(h, c->h_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *Sg = h[0];
    if (cos_sum)
        *cos_sum = h[1];
    return DWF_OK;
}

// Pseudofermion action and force on slot 0: eta = (D D^dag)^-1 phi (warm
// start from h_eta when has_guess), S = Re<phi, eta>, xi = D^dag eta,
// h_force += F_pf. Domain wall: the solve must converge
// (pseudofermion.hpp:32-41). Wilson: started from zero and accepted when the
// FP64 residual is within 20 tol (wilson/include/cg_solver.hpp:53-78).
int pf_force(dwf_ctx* c, const double2* phi, int has_guess, double rtol, int maxiter, int solver,
             double* Spf, dwf_solve_info* info_out)
{
    const bool wilson = c->kind == 1;
    dwf_solve_info info{};
    const int conf0 = 0;
    int st = solve_batch(c, DWF_OP_DDDAG, 1, &conf0, phi, c->h_eta, wilson ? 0 : has_guess, rtol,
                         maxiter, solver, wilson ? 1 : 0, &info);
    if (st)
        return st;
    if (info_out)
        *info_out = info;
    if (wilson)
    {
        if (!std::isfinite(info.true_relres) || info.true_relres > 20.0 * rtol)
        {
            char msg[160];
            std::snprintf(msg, sizeof msg, "pseudofermion CG failed: iterations=%d, residual=%e",
                          info.iterations, info.true_relres);
            return ctx_fail(c, DWF_NOT_CONVERGED, msg);
        }
    }
    else if (info.status != DWF_OK)
        return ctx_fail(c, info.status == DWF_ZERO_DENOM ? DWF_ZERO_DENOM : DWF_NOT_CONVERGED,
                        info.status == DWF_ZERO_DENOM ? "CG encountered a zero denominator"
                                                      : "Pseudofermion CG failed to converge");
    const long n = c->fsz();
    dot_re_kernel<<<kRedBlocks, 256, 0, c->stream>>>(phi, c->h_eta, n, c->h_part);
    finish_sum_kernel<<<1, 64, 0, c->stream>>>(c->h_part, kRedBlocks, 1, c->h_scal + 2);
    st = apply_dev(c, DWF_OP_DDAG, 1, nullptr, 0, c->h_eta, c->h_xi, 64);
    if (st)
        return st;
    pf_force_kernel<<<std::max(1, (2 * c->L.V + 255) / 256), 256, 0, c->stream>>>(
        c->L, c->h_eta, c->h_xi, c->U64, c->h_force);
    CK(cudaGetLastError());
    c->launches += 3;
    CK(cudaMemcpyAsync(Spf, c->h_scal + 2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int kinetic(dwf_ctx* c, double* K)
{
    kinetic_kernel<<<kRedBlocks, 256, 0, c->stream>>>(c->h_mom, c->usz(), c->h_part);
    finish_sum_kernel<<<1, 64, 0, c->stream>>>(c->h_part, kRedBlocks, 1, c->h_scal + 3);
    CK(cudaGetLastError());
    c->launches += 2;
    CK(cudaMemcpyAsync(K, c->h_scal + 3, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int kick(dwf_ctx* c, double coef)
{
    const long n = c->usz();
    kick_kernel<<<int(std::min<long>((n + 255) / 256, 1024)), 256, 0, c->stream>>>(c->h_mom, c->h_force, coef, n);
    CK(cudaGetLastError());
    c->launches += 1;
    return DWF_OK;
}

int drift(dwf_ctx* c, double eps, int wrap)
{
    const long n = c->usz();
    drift_kernel<<<int(std::min<long>((n + 255) / 256, 1024)), 256, 0, c->stream>>>(c->theta, c->h_mom, eps, wrap, n, c->U64, c->U32);
    CK(cudaGetLastError());
    c->launches += 1;
    return DWF_OK;
}

int begin(dwf_ctx* c, const double* theta)
{
    if (!c || !theta)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    int st = set_gauge(c, 1, theta, cudaMemcpyHostToDevice);
    if (st)
        return st;
    return ensure_hmc(c);
}

int validate(dwf_ctx* c, const dwf_hmc_params* hp)
{
    if (!hp || hp->steps < 1 || !(hp->epsilon == hp->epsilon) || hp->maxiter < 0 ||
        !(hp->rtol >= 0.0) || (hp->solver != DWF_SOLVER_CG64 && hp->solver != DWF_SOLVER_MIXED))
        return ctx_fail(c, DWF_BAD_ARG, "hmc: bad parameters");
    return DWF_OK;
}

}  // namespace

extern "C" {

int dwf_gauge_action_force(dwf_ctx* c, const double* theta, double* action, double* force)
{
    int st = begin(c, theta);
    if (st)
        return st;
    double sg = 0.0;
    st = gauge_force(c, &sg, nullptr);
    if (st)
        return st;
    if (action)
        *action = sg;
    if (force)
    {
        CK(cudaMemcpyAsync(force, c->h_force, c->usz() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return DWF_OK;
}

int dwf_average_plaquette(dwf_ctx* c, const double* theta, double* plaquette)
{
    int st = begin(c, theta);
    if (st)
        return st;
    double sg = 0.0, cs = 0.0;
    st = gauge_force(c, &sg, &cs);
    if (st)
        return st;
    *plaquette = cs / double(c->L.V);
    return DWF_OK;
}

int dwf_pf_action_force(dwf_ctx* c, const double* theta, const double* phi, const double* eta_guess,
                        double rtol, int maxiter, int solver, double* action, double* force,
                        double* eta_out, dwf_solve_info* info)
{
    if (!phi)
        return DWF_BAD_ARG;
    int st = begin(c, theta);
    if (st)
        return st;
    const size_t fb = c->fsz() * sizeof(double2);
    CK(cudaMemcpyAsync(c->h_phi, phi, fb, cudaMemcpyHostToDevice, c->stream));
    if (eta_guess)
        CK(cudaMemcpyAsync(c->h_eta, eta_guess, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->h_force, 0, c->usz() * sizeof(double), c->stream));
    double spf = 0.0;
    st = pf_force(c, c->h_phi, eta_guess != nullptr, rtol, maxiter, solver, &spf, info);
    if (st)
        return st;
    if (action)
        *action = spf;
    if (force)
        CK(cudaMemcpyAsync(force, c->h_force, c->usz() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (eta_out)
        CK(cudaMemcpyAsync(eta_out, c->h_eta, fb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

// One domain-wall trajectory (domain_wall/generate_configs.cpp:56-160): phi = D chi,
// leapfrog with half kicks at both ends, warm-started pseudofermion solves, no
// angle wrapping, H from the actions of the last force evaluation.
int dwf_hmc_trajectory(dwf_ctx* c, const dwf_hmc_params* hp, const double* theta0,
                       const double* chi, const double* mom, double* theta_out,
                       dwf_traj_info* info)
{
    if (!c || !chi || !mom || !theta_out || c->kind != 0)
        return DWF_BAD_ARG;
    int st = validate(c, hp);
    if (st)
        return st;
    if ((st = begin(c, theta0)))
        return st;
    const size_t fb = c->fsz() * sizeof(double2);
    const size_t gb = c->usz() * sizeof(double);
    CK(cudaMemcpyAsync(c->h_chi, chi, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->h_mom, mom, gb, cudaMemcpyHostToDevice, c->stream));
    if ((st = apply_dev(c, DWF_OP_D, 1, nullptr, 0, c->h_chi, c->h_phi, 64)))
        return st;
    dwf_traj_info I{};
    double sg = 0.0, spf = 0.0, k0 = 0.0;
    dwf_solve_info si{};
    if ((st = gauge_force(c, &sg, nullptr)))
        return st;
    if ((st = pf_force(c, c->h_phi, 0, hp->rtol, hp->maxiter, hp->solver, &spf, &si)))
        return st;
    I.cg_iterations += si.iterations;
    I.solves += 1;
    if ((st = kinetic(c, &k0)))
        return st;
    I.kinetic0 = k0;
    I.H0 = k0 + sg + spf;
    if ((st = kick(c, 0.5 * hp->epsilon)))
        return st;
    for (int step = 0; step < hp->steps; ++step)
    {
        if ((st = drift(c, hp->epsilon, 0)))
            return st;
        if ((st = gauge_force(c, &sg, nullptr)))
            return st;
        if ((st = pf_force(c, c->h_phi, 1, hp->rtol, hp->maxiter, hp->solver, &spf, &si)))
            return st;
        I.cg_iterations += si.iterations;
        I.solves += 1;
        if (step != hp->steps - 1 && (st = kick(c, hp->epsilon)))
            return st;
    }
    if ((st = kick(c, 0.5 * hp->epsilon)))
        return st;
    double k1 = 0.0;
    if ((st = kinetic(c, &k1)))
        return st;
    I.kinetic = k1;
    I.S_gauge = sg;
    I.S_pf = spf;
    I.H = k1 + sg + spf;
    I.dH = I.H - I.H0;
    double tmp = 0.0, cs = 0.0;
    if ((st = gauge_force(c, &tmp, &cs)))
        return st;
    I.plaquette = cs / double(c->L.V);
    I.acceptance_probability = std::min(std::exp(-I.dH), 1.0);
    I.status = DWF_OK;
    CK(cudaMemcpyAsync(theta_out, c->theta, gb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (info)
        *info = I;
    return DWF_OK;
}

// ---------------------------------------------------------------------------
// Wilson
// ---------------------------------------------------------------------------
int wil_ctx_create(const wil_params* p, dwf_ctx** out)
{
    if (!p || !out)
        return DWF_BAD_ARG;
    *out = nullptr;
    if (p->Nt < 1 || p->Nx < 1 || long(p->Nt) * p->Nx > (1L << 30))
        return DWF_BAD_ARG;
    dwf_ctx* c = new dwf_ctx();
    c->kind = 1;
    c->L.Nt = p->Nt;
    c->L.Nx = p->Nx;
    c->L.Ls = 1;
    c->L.V = p->Nt * p->Nx;
    c->L.nsite = c->L.V;
    c->L.diag = 2.0 + p->m0;
    c->L.mf = 0.0;
    c->L.bct = p->bc_t;
    c->L.bcx = p->bc_x;
    c->L.fifth = 0;
    c->beta = p->beta;
    const int st = dwfb_ctx_init(c, p->device);
    if (st)
    {
        dwf_ctx_destroy(c);
        return st;
    }
    *out = c;
    return DWF_OK;
}

// solve_CGNR (wilson/include/cg_solver.hpp:19-51): x = (D^dag D)^-1 D^dag source,
// Eigen's stopping rule, then the FP64 normal and Dirac residuals; status
// DWF_NOT_CONVERGED when the normal residual exceeds 20 tol or is not finite.
int wil_solve_cgnr(dwf_ctx* c, const double* theta, const double* source, double tol,
                   int maxiter, int solver, double* x, double* info3)
{
    if (!c || c->kind != 1 || !theta || !source || !x)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    int st = set_gauge(c, 1, theta, cudaMemcpyHostToDevice);
    if (st)
        return st;
    dwf_solve_info info{};
    st = dwf_propagators(c, 1, nullptr, source, x, tol, maxiter, solver, &info);
    if (st)
        return st;
    if (info3)
    {
        info3[0] = info.iterations;
        info3[1] = info.true_relres;
        info3[2] = info.dirac_relres;
    }
    if (!std::isfinite(info.true_relres) || info.true_relres > 20.0 * tol)
    {
        char msg[200];
        std::snprintf(msg, sizeof msg, "CGNR failed: iterations=%d, normal residual=%e, D residual=%e",
                      info.iterations, info.true_relres, info.dirac_relres);
        return ctx_fail(c, DWF_NOT_CONVERGED, msg);
    }
    return DWF_OK;
}

// solve_DDdag (wilson/include/cg_solver.hpp:53-78).
int wil_solve_dddag(dwf_ctx* c, const double* theta, const double* phi, double tol, int maxiter,
                    int solver, double* eta, double* residual)
{
    if (!c || c->kind != 1 || !theta || !phi || !eta)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    int st = set_gauge(c, 1, theta, cudaMemcpyHostToDevice);
    if (st)
        return st;
    dwf_solve_info info{};
    st = dwf_cg(c, DWF_OP_DDDAG, 0, phi, eta, 0, tol, maxiter, solver, &info);
    if (st != DWF_OK && st != DWF_NOT_CONVERGED)
        return st;
    if (residual)
        *residual = info.true_relres;
    if (!std::isfinite(info.true_relres) || info.true_relres > 20.0 * tol)
    {
        char msg[160];
        std::snprintf(msg, sizeof msg, "pseudofermion CG failed: iterations=%d, residual=%e",
                      info.iterations, info.true_relres);
        return ctx_fail(c, DWF_NOT_CONVERGED, msg);
    }
    return DWF_OK;
}

// hmc_step (wilson/include/gauge.hpp:132-180) with the momenta, chi and the
// Metropolis uniform supplied by the caller in the reference's draw order.
// Angles are wrapped into [-pi, pi) on every drift; the last kick is halved
// inside the loop; the final actions are those of the configuration reached
// (the reference recomputes them with one more solve at the same angles,
// which gives the same values).
int wil_hmc_step(dwf_ctx* c, const dwf_hmc_params* hp, const double* theta_old,
                 const double* mom, const double* chi, double u, double* theta_out,
                 dwf_traj_info* info)
{
    if (!c || c->kind != 1 || !mom || !chi || !theta_out || !theta_old)
        return DWF_BAD_ARG;
    int st = validate(c, hp);
    if (st)
        return st;
    if ((st = begin(c, theta_old)))
        return st;
    const size_t fb = c->fsz() * sizeof(double2);
    const size_t gb = c->usz() * sizeof(double);
    CK(cudaMemcpyAsync(c->h_chi, chi, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->h_mom, mom, gb, cudaMemcpyHostToDevice, c->stream));
    if ((st = apply_dev(c, DWF_OP_D, 1, nullptr, 0, c->h_chi, c->h_phi, 64)))
        return st;
    dwf_traj_info I{};
    dwf_solve_info si{};
    double sg = 0.0, spf = 0.0, k0 = 0.0;
    if ((st = gauge_force(c, &sg, nullptr)))
        return st;
    if ((st = pf_force(c, c->h_phi, 0, hp->rtol, hp->maxiter, hp->solver, &spf, &si)))
        return st;
    I.cg_iterations += si.iterations;
    I.solves += 1;
    if ((st = kinetic(c, &k0)))
        return st;
    I.kinetic0 = k0;
    I.H0 = k0 + sg + spf;
    if ((st = kick(c, 0.5 * hp->epsilon)))
        return st;
    for (int step = 0; step < hp->steps; ++step)
    {
        if ((st = drift(c, hp->epsilon, 1)))
            return st;
        if ((st = gauge_force(c, &sg, nullptr)))
            return st;
        if ((st = pf_force(c, c->h_phi, 0, hp->rtol, hp->maxiter, hp->solver, &spf, &si)))
            return st;
        I.cg_iterations += si.iterations;
        I.solves += 1;
        const double factor = (step == hp->steps - 1) ? 0.5 : 1.0;
        if ((st = kick(c, factor * hp->epsilon)))
            return st;
    }
    double k1 = 0.0;
    if ((st = kinetic(c, &k1)))
        return st;
    I.kinetic = k1;
    I.S_gauge = sg;
    I.S_pf = spf;
    I.H = k1 + sg + spf;
    I.dH = I.H - I.H0;
    I.acceptance_probability = std::min(1.0, std::exp(-I.dH));
    I.accepted = (u < I.acceptance_probability) ? 1 : 0;
    if (I.accepted)
    {
        CK(cudaMemcpyAsync(theta_out, c->theta, gb, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    else
    {
        std::copy(theta_old, theta_old + c->usz(), theta_out);
        if ((st = set_gauge(c, 1, theta_old, cudaMemcpyHostToDevice)))
            return st;
    }
    double tmp = 0.0, cs = 0.0;  // plaquette of the configuration returned
    if ((st = gauge_force(c, &tmp, &cs)))
        return st;
    I.plaquette = cs / double(c->L.V);
    I.status = DWF_OK;
    if (info)
        *info = I;
    return DWF_OK;
}

}  // extern "C"
