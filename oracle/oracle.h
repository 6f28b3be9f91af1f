/* CPU oracle for the Wilson / domain-wall hot path (TEST INFRASTRUCTURE ONLY).
 *
 * A plain C++ restatement of the reference's arithmetic with every lattice
 * parameter passed explicitly (the reference reads them from ./parameters.txt
 * at static-initialisation time). Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library, and only to check GPU results
 * or as the timed CPU baseline; the product never calls it.
 *
 * Conventions (identical to the reference):
 *   gauge theta   : double[2*Nt*Nx], index (mu*Nt + t)*Nx + x        (domain_wall/include/indexing.hpp:10-13)
 *   DWF fermion   : complex<double>[Ls*Nt*Nx*2] interleaved re,im,
 *                   index ((s*Nt + t)*Nx + x)*2 + spin              (domain_wall/include/indexing.hpp:5-8)
 *   Wilson fermion: complex<double>[Nt*Nx*2], index (t*Nx + x)*2 + spin (wilson/include/indexing.hpp:5-8)
 * Complex arrays are passed as double* with re,im interleaved.
 * Status codes: 0 ok, 1 not converged, 2 zero denominator, 6 bad argument.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
    int Nt, Nx, Ls;
    double M5, mf;
} orc_dwf_params;

typedef struct
{
    int Nt, Nx;
    double m0, bc_t, bc_x;
} orc_wil_params;

enum { ORC_D = 0, ORC_DDAG = 1, ORC_DDDAG = 2, ORC_DDAGD = 3 };

/* ---- domain wall --------------------------------------------------------- */
void orc_dwf_apply(const orc_dwf_params* p, int op, const double* theta, const double* in,
                   double* out);
int orc_dwf_cg(const orc_dwf_params* p, int op, const double* theta, const double* b,
               const double* guess, double rtol, int maxiter, double* x, int* iters,
               double* relres);
int orc_dwf_pf_action_force(const orc_dwf_params* p, const double* theta, const double* phi,
                            const double* guess, double rtol, int maxiter, double* action,
                            double* force, double* eta, int* iters, double* relres);
void orc_gauge_action_force(int Nt, int Nx, double beta, const double* theta, double* action,
                            double* force);
double orc_average_plaquette(int Nt, int Nx, const double* theta);
/* out6 = {dH, H0, H, S_gauge_final, S_pf_final, total CG iterations} */
int orc_dwf_trajectory(const orc_dwf_params* p, double beta, double eps, int nsteps, double rtol,
                       int maxiter, const double* theta0, const double* chi, const double* mom,
                       double* theta_out, double* out6);
/* psi_out: 2 propagators (source spin 0, 1), each Ndof complex; info: per spin
 * {iterations, normal relres, Dirac residual, converged} */
int orc_dwf_wall_propagator(const orc_dwf_params* p, const double* theta, int t_src, double rtol,
                            int maxiter, double* psi_out, double* info8);
int orc_dwf_cpp_cj5(const orc_dwf_params* p, const double* theta, double rtol, int maxiter,
                    double* cpp, double* cj5);
int orc_dwf_momentum_cpp(const orc_dwf_params* p, const double* theta, int max_momentum,
                         double rtol, int maxiter, double* out);
int orc_dwf_loop(const orc_dwf_params* p, const double* theta, unsigned long long seed,
                 int nnoise, double rtol, int maxiter, double* loop);

/* ---- random streams (libstdc++ engines, as the reference draws them) ------ */
void orc_rng_z4(unsigned long long seed, long n, int* digits);
void orc_rng_normals(unsigned long long seed, long n, double* out);
/* DWF generator order per trajectory: chi[Ndof] (imag drawn first), mom[2V], u */
void orc_dwf_draws(unsigned long long seed, int ntraj, int ndof, int ngauge, double* chi,
                   double* mom, double* u);
/* Wilson hmc_step order per trajectory: mom[2V], chi[Ntot] (imag drawn first), u */
void orc_wil_draws(unsigned long long seed, int ntraj, int ntot, int ngauge, double* mom,
                   double* chi, double* u);

/* ---- Wilson --------------------------------------------------------------- */
void orc_wil_apply(const orc_wil_params* p, int op, const double* theta, const double* in,
                   double* out);
/* Jacobi-preconditioned CG on the assembled normal matrix (op ORC_DDDAG or ORC_DDAGD),
 * started from zero, stopping at |r|^2 < tol^2 |b|^2. */
int orc_wil_cg(const orc_wil_params* p, int op, const double* theta, const double* b, double tol,
               int maxiter, double* x, int* iters, double* relres);
/* info3 = {iterations, normal residual, Dirac residual}; status 1 if the 20*tol check fails */
int orc_wil_solve_cgnr(const orc_wil_params* p, const double* theta, const double* source,
                       double tol, int maxiter, double* x, double* info3);
int orc_wil_solve_dddag(const orc_wil_params* p, const double* theta, const double* phi,
                        double tol, int maxiter, double* eta, double* residual);
int orc_wil_pf_action_force(const orc_wil_params* p, const double* theta, const double* phi,
                            double tol, int maxiter, double* action, double* force);
/* info3 = {dH, acceptance probability, accepted}; theta_out = accepted ? new : old */
int orc_wil_hmc_step(const orc_wil_params* p, double beta, double eps, int nsteps, double tol,
                     int maxiter, const double* theta_old, const double* mom, const double* chi,
                     double u, double* theta_out, double* info3);
int orc_wil_correlator(const orc_wil_params* p, const double* theta, int src_t, int src_x,
                       double tol, int maxiter, double* corr);

#ifdef __cplusplus
}
#endif
