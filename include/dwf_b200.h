/* dwf_b200.h -- C ABI of the B200 (sm_100a) implementation of the lattice
 * study's dynamical-fermion hot path: the Wilson and domain-wall Dirac
 * operators, CG on the normal operator, the pseudofermion force and link
 * update inside HMC, and the propagator solves with their meson contractions.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns an int status (dwf_status). Host layouts are the reference's:
 *
 *   gauge theta  double[2*Nt*Nx]          index (mu*Nt + t)*Nx + x
 *                                           (domain_wall/include/indexing.hpp:10-13,
 *                                            wilson/include/indexing.hpp:9-12)
 *   DWF fermion  complex<double>[Ls*Nt*Nx*2], interleaved (re, im),
 *                index ((s*Nt + t)*Nx + x)*2 + spin  (domain_wall/include/indexing.hpp:5-8)
 *   Wilson       complex<double>[Nt*Nx*2], index (t*Nx + x)*2 + spin
 *                                           (wilson/include/indexing.hpp:5-8)
 *
 * Entry points whose name ends in _dev take device pointers (laid out the
 * same way, one right-hand side after another) and run on the context's
 * stream (dwf_stream); the caller orders that stream against the streams that
 * produce the inputs and consume the outputs (e.g. cudaStreamWaitEvent both
 * ways). The others take host pointers, copy, and return when done.
 *
 * Ownership: the caller owns every buffer it passes. A context owns its
 * device memory and stream. One context per host thread: a context is not
 * safe for concurrent use, distinct contexts are independent.
 */
#ifndef DWF_B200_H
#define DWF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The C++ host layer maps them to the reference's
 * std::runtime_error messages (e.g. "CG encountered a zero denominator",
 * domain_wall/include/cg_solver.hpp:45-46). */
typedef enum
{
    DWF_OK = 0,
    DWF_NOT_CONVERGED = 1,
    DWF_ZERO_DENOM = 2,
    DWF_NONFINITE = 3,
    DWF_CUDA_ERROR = 4,
    DWF_TIMEOUT = 5,
    DWF_BAD_ARG = 6
} dwf_status;

/* Operators (domain_wall/include/dwf_operator.hpp:15,94,173,178). */
typedef enum
{
    DWF_OP_D = 0,
    DWF_OP_DDAG = 1,
    DWF_OP_DDDAG = 2, /* D D^dag  (pseudofermion solve) */
    DWF_OP_DDAGD = 3  /* D^dag D  (propagator / CGNR solve) */
} dwf_op;

/* Solver paths. */
typedef enum
{
    /* The reference algorithm in FP64: unpreconditioned CG, stop when the
     * recursive residual satisfies |r|/|b| <= rtol
     * (domain_wall/include/cg_solver.hpp:17-64). */
    DWF_SOLVER_CG64 = 0,
    /* FP32 inner CG iterations with FP64 reliable updates (true residual
     * recomputed in FP64); converged only when the FP64 true residual meets
     * rtol. Falls back to DWF_SOLVER_CG64 from its current iterate if the
     * true residual stalls. */
    DWF_SOLVER_MIXED = 1,
    /* Propagator solves (dwf_propagators, dwf_measure): even-odd
     * (4-D checkerboard) Schur-complement preconditioned mixed CG for
     * D x = src, then, where the FP64 residual of the full D^dag D misses rtol,
     * DWF_SOLVER_CG64 on the full D^dag D from that x, so the reference's
     * stopping rule on the full normal equation decides. Needs even
     * Nt, Nx and 3 - M5 >= 1 (else it runs DWF_SOLVER_MIXED); elsewhere it is
     * DWF_SOLVER_MIXED. */
    DWF_SOLVER_EO_MIXED = 2,
    /* Propagator solves with the learned preconditioner (no counterpart in the
     * reference; needs dwf_lp_init, normally followed by dwf_lp_train): FP64
     * defect correction around an FP32 flexible GCR (dwf_lp_set_krylov) on
     * D x = src, right-preconditioned by the gauge-equivariant network N ~ D^-1 (BF16 channel
     * mixing, FP32 accumulation); the reference's stopping rule
     * |D^dag (D x - src)| <= rtol |D^dag src| is checked on the FP64 true
     * residual after each inner solve. A right-hand side whose true residual
     * falls by less than a factor 2 in a cycle continues with DWF_SOLVER_MIXED
     * (CG on D^dag D) from its iterate (info.fallback = 1). */
    DWF_SOLVER_LEARNED = 3
} dwf_solver;

/* Domain-wall context parameters: the parameters.txt keys dwf.Nt, dwf.Nx,
 * dwf.N5, dwf.M5, dwf.mf, dwf.beta (domain_wall/include/parameters.hpp:7-20). */
typedef struct
{
    int Nt, Nx, Ls;
    double M5, mf;
    double beta;
    int device; /* CUDA device ordinal */
} dwf_params;

/* Per-solve report. */
typedef struct
{
    int iterations;      /* CG iterations, counted as the reference counts them */
    int converged;       /* 1 if the stopping rule was met */
    int status;          /* dwf_status of this right-hand side */
    int solver;          /* dwf_solver path that produced x */
    double relres;       /* recursive residual |r|/|b| at exit */
    double true_relres;  /* FP64 |b - A x| / |b| recomputed after the solve */
    int reliable_updates;/* FP64 residual replacements (mixed path) */
    int fallback;        /* 1 if the mixed path fell back to FP64 CG */
    double dirac_relres; /* propagator solves: |D x - src| / |src| (correlator.hpp:225-227); else 0 */
    int schur_iterations;/* DWF_SOLVER_EO_MIXED: iterations of the even-odd stage (included
                            in `iterations`); DWF_SOLVER_LEARNED: preconditioned BiCGStab
                            iterations (2 network and 2 D applications each); else 0 */
} dwf_solve_info;

typedef struct dwf_ctx dwf_ctx;

/* ---- context ------------------------------------------------------------ */
int dwf_ctx_create(const dwf_params* params, dwf_ctx** out);
int dwf_ctx_destroy(dwf_ctx* ctx);
const char* dwf_status_string(int status);
/* Last error message recorded on this context ("" if none). */
const char* dwf_last_error(const dwf_ctx* ctx);
/* Limit (ns) for every bounded wait inside persistent kernels (default 5 s). */
int dwf_set_wait_limit(dwf_ctx* ctx, uint64_t nanoseconds);
/* Synchronise the context stream. */
int dwf_sync(dwf_ctx* ctx);
/* The context's cudaStream_t, as void*. */
void* dwf_stream(dwf_ctx* ctx);

/* ---- gauge field ---------------------------------------------------------- */
/* Upload nconf configurations (host, nconf * 2*Nt*Nx doubles). The context
 * caches link phases U = exp(i theta) in FP64 and FP32
 * (domain_wall/include/dwf_operator.hpp:10-13). */
int dwf_set_gauge(dwf_ctx* ctx, int nconf, const double* theta);
/* Same from a device buffer. */
int dwf_set_gauge_dev(dwf_ctx* ctx, int nconf, const double* theta_dev);

/* ---- operators ---------------------------------------------------------- */
/* out = op(in) for nrhs fields, all on configuration `conf`
 * (apply_D / apply_D_dagger / apply_DD_dagger / apply_D_dagger_D,
 *  domain_wall/include/dwf_operator.hpp:15-181). */
int dwf_apply(dwf_ctx* ctx, int op, int conf, const double* in, double* out, int nrhs);
/* Device version; precision 64 (complex<double>) or 32 (complex<float>).
 * Both fields must start on a 16-byte boundary (DWF_BAD_ARG otherwise). */
int dwf_apply_dev(dwf_ctx* ctx, int op, int conf, const void* in_dev, void* out_dev, int nrhs,
                  int precision);

/* ---- solver ----------------------------------------------------------------- */
/* Solve A x = b with A = op (DWF_OP_DDDAG or DWF_OP_DDAGD) on configuration
 * `conf`. x is read as the initial guess when has_guess != 0 (the reference's
 * initial_guess pointer), else started from zero. Host pointers.
 * (conjugate_gradient, domain_wall/include/cg_solver.hpp:17-64) */
int dwf_cg(dwf_ctx* ctx, int op, int conf, const double* b, double* x, int has_guess,
           double rtol, int maxiter, int solver, dwf_solve_info* info);
/* Batched device version: nrhs right-hand sides, rhs k on configuration
 * rhs_conf[k] (host array; NULL = all on configuration 0), solved together
 * in one persistent launch with per-right-hand-side convergence.
 * info: host array of nrhs reports. */
int dwf_cg_batch_dev(dwf_ctx* ctx, int op, int nrhs, const int* rhs_conf, const void* b_dev,
                     void* x_dev, int has_guess, double rtol, int maxiter, int solver,
                     dwf_solve_info* info);
/* Host-buffer version of dwf_cg_batch_dev. */
int dwf_cg_batch(dwf_ctx* ctx, int op, int nrhs, const int* rhs_conf, const double* b, double* x,
                 int has_guess, double rtol, int maxiter, int solver, dwf_solve_info* info);

/* ---- propagators -------------------------------------------------------------- */
/* The analyzers' propagator solve for nrhs sources at once: x = (D^dag D)^-1 D^dag src,
 * i.e. rhs = apply_D_dagger(theta, source) followed by conjugate_gradient on
 * apply_D_dagger_D from zero (domain_wall/include/correlator.hpp:77-79, :139-142,
 * :213-220). info[k].dirac_relres = |D x - src| / |src|. Host buffers. With
 * DWF_SOLVER_EO_MIXED on the cluster solver and nrhs of at least two of its
 * waves (the right-hand sides its resident clusters solve at once), the batch
 * runs in two chunks of whole waves, the copies of each chunk on a second
 * stream overlapping the solve of the other (page-locked buffers let them
 * overlap); each source's Schur solve is the one a single batch would run,
 * and the full-lattice check is decided per chunk. */
int dwf_propagators(dwf_ctx* ctx, int nrhs, const int* rhs_conf, const double* src, double* x,
                    double rtol, int maxiter, int solver, dwf_solve_info* info);
/* Device-buffer version. */
int dwf_propagators_dev(dwf_ctx* ctx, int nrhs, const int* rhs_conf, const void* src_dev,
                        void* x_dev, double rtol, int maxiter, int solver, dwf_solve_info* info);

/* ---- HMC ------------------------------------------------------------------ */
/* Leapfrog parameters. Domain wall: epsilon = dwf.epsilon, steps =
 * dwf.leapfrog_steps, rtol/maxiter = dwf.pseudofermion_rtol/_maxiter.
 * Wilson: epsilon = wilson.trajectory_length / wilson.hmc_steps, steps =
 * wilson.hmc_steps, rtol/maxiter = wilson.force_cg_tolerance/_max_iterations. */
typedef struct
{
    double epsilon;
    int steps;
    double rtol;
    int maxiter;
    int solver; /* dwf_solver used for the pseudofermion solves */
} dwf_hmc_params;

typedef struct
{
    double dH, H0, H;        /* Hamiltonian change, initial and final (FP64) */
    double S_gauge, S_pf;    /* actions at the final configuration */
    double kinetic0, kinetic;
    double plaquette;        /* average plaquette: proposal (domain wall), result (Wilson) */
    double acceptance_probability; /* min(1, exp(-dH)) */
    int accepted;            /* Wilson only: u < acceptance_probability */
    int solves;              /* pseudofermion solves performed */
    long cg_iterations;      /* summed over those solves */
    int status;
} dwf_traj_info;

/* Gauge action beta sum(1 - cos P) and force on host theta
 * (gauge_action_force, domain_wall/include/gauge.hpp:26-62; wilson/include/gauge.hpp:38-62).
 * Uses the context's beta. force: host double[2*Nt*Nx] or NULL. */
int dwf_gauge_action_force(dwf_ctx* ctx, const double* theta, double* action, double* force);
/* average_plaquette (domain_wall/include/gauge.hpp:64-73; wilson/include/gauge.hpp:29-36). */
int dwf_average_plaquette(dwf_ctx* ctx, const double* theta, double* plaquette);
/* Pseudofermion action S = Re<phi, eta>, eta = (D D^dag)^-1 phi, and its force
 * (pseudofermion_action_force, domain_wall/include/pseudofermion.hpp:22-166;
 * wilson/include/gauge.hpp:68-122). eta_guess may be NULL (domain wall warm start;
 * Wilson always starts from zero). force, eta_out may be NULL. */
int dwf_pf_action_force(dwf_ctx* ctx, const double* theta, const double* phi,
                        const double* eta_guess, double rtol, int maxiter, int solver,
                        double* action, double* force, double* eta_out, dwf_solve_info* info);
/* One domain-wall HMC trajectory from theta0 with the heat-bath draws chi
 * (Ndof complex) and mom (2*Nt*Nx) supplied by the caller: phi = D chi, leapfrog,
 * proposal in theta_out, dH in info (domain_wall/generate_configs.cpp:56-160).
 * The Metropolis test (:158-169) is the caller's, with its own uniform draw. */
int dwf_hmc_trajectory(dwf_ctx* ctx, const dwf_hmc_params* hp, const double* theta0,
                       const double* chi, const double* mom, double* theta_out,
                       dwf_traj_info* info);

/* ---- Wilson ------------------------------------------------------------------ */
/* Wilson context: parameters.txt keys wilson.Nt, wilson.Nx, wilson.m0, wilson.beta,
 * wilson.time_boundary_sign, wilson.space_boundary_sign
 * (wilson/include/parameters.hpp:6-27). The context works with every dwf_*
 * entry point above (operators act on Wilson fields, Ls = 1); its solves use
 * the stopping rule of the reference's Eigen ConjugateGradient,
 * |r|^2 < tol^2 |b|^2 (wilson/include/cg_solver.hpp:24-31). */
typedef struct
{
    int Nt, Nx;
    double m0, beta;
    double bc_t, bc_x;
    int device;
} wil_params;

int wil_ctx_create(const wil_params* params, dwf_ctx** out);
/* solve_CGNR (wilson/include/cg_solver.hpp:19-51). info3 = {iterations, normal
 * residual, Dirac residual}; DWF_NOT_CONVERGED (with the reference's message in
 * dwf_last_error) when the normal residual exceeds 20 tol. */
int wil_solve_cgnr(dwf_ctx* ctx, const double* theta, const double* source, double tol,
                   int maxiter, int solver, double* x, double* info3);
/* solve_DDdag (wilson/include/cg_solver.hpp:53-78). */
int wil_solve_dddag(dwf_ctx* ctx, const double* theta, const double* phi, double tol, int maxiter,
                    int solver, double* eta, double* residual);
/* hmc_step (wilson/include/gauge.hpp:124-180) with mom, chi and the uniform u
 * drawn by the caller (order: mom, chi, u). theta_out = accepted ? new : old. */
int wil_hmc_step(dwf_ctx* ctx, const dwf_hmc_params* hp, const double* theta_old,
                 const double* mom, const double* chi, double u, double* theta_out,
                 dwf_traj_info* info);

/* ---- measurements ------------------------------------------------------------ */
/* Per-configuration source set: boundary point sources at x = 0 and boundary
 * wall sources, each at source times t_k = k*Nt/n (k < n) for both source
 * spins, and n_noise complex Z4 boundary-noise vectors. n_point_times =
 * n_wall_times = 2 gives the reference's {0, Nt/2}
 * (domain_wall/include/correlator.hpp:120, :251). */
typedef struct
{
    int n_point_times;
    int n_wall_times;
    int n_noise;      /* eta.noise_vectors */
    int max_momentum; /* analysis.max_momentum (0..Nx/2) */
    double rtol;      /* dwf.propagator_rtol */
    int maxiter;      /* dwf.propagator_maxiter */
    int solver;       /* dwf_solver */
} dwf_measure_params;

/* All propagators of nconf configurations in one batched solve, then the
 * contractions (domain_wall/include/correlator.hpp:27-310):
 *   cpp, cj5 : [nconf][Nt]  C_PP and C_J5 from the wall sources (compute_CPP_CJ5)
 *   loop     : [nconf][Nt*Nx] complex, the Z4 loop density
 *              (estimate_pseudoscalar_loop_density)
 *   mom_cpp  : [nconf][max_momentum+1][Nt] from the point sources (compute_momentum_CPP)
 * z4: [nconf][n_noise][Nt][Nx][2] digits 0..3 drawn by the caller in the
 * reference's order (dwf_z4_digits with seed eta.random_seed + 104729*config,
 * domain_wall/analyze_configs.cpp:66-68). Output pointers may be NULL.
 * info: [nconf * (2*n_point_times + 2*n_wall_times + n_noise)] or NULL,
 * right-hand sides ordered point, wall, noise within each configuration. */
int dwf_measure(dwf_ctx* ctx, const dwf_measure_params* mp, int nconf, const double* thetas,
                const signed char* z4, double* cpp, double* cj5, double* loop, double* mom_cpp,
                dwf_solve_info* info);
/* pseudoscalar_correlator (wilson/include/correlator.hpp:10-40) for nconf
 * configurations: corr [nconf][Nt]. DWF_NOT_CONVERGED (reference message in
 * dwf_last_error) if any solve misses the 20*tol check of solve_CGNR.
 * info: [2*nconf] or NULL. */
int wil_pseudoscalar_correlator(dwf_ctx* ctx, int nconf, const double* thetas, int src_t,
                                int src_x, double tol, int maxiter, int solver, double* corr,
                                dwf_solve_info* info);

/* ---- host random streams ----------------------------------------------------- */
/* The reference draws from std::mt19937_64 with std::normal_distribution<double>,
 * std::uniform_real_distribution<double>(0, 1) (domain_wall/generate_configs.cpp:23-25,
 * wilson/include/gauge.hpp:16-18) and std::uniform_int_distribution<int>(0, 3)
 * (domain_wall/include/correlator.hpp:35-36); these reproduce those streams. */
typedef struct dwf_rng dwf_rng;
int dwf_rng_create(uint64_t seed, dwf_rng** out);
int dwf_rng_destroy(dwf_rng* rng);
int dwf_rng_normals(dwf_rng* rng, long n, double* out);
int dwf_rng_uniform(dwf_rng* rng, double* out);
/* n complex entries Complex(normal, normal)/sqrt(2), imaginary part drawn
 * first, as the reference's chi (generate_configs.cpp:58-62, gauge.hpp:138-140). */
int dwf_rng_pseudofermion(dwf_rng* rng, long n, double* chi);
/* n Z4 digits from mt19937_64(seed) (correlator.hpp:35-58). */
int dwf_z4_digits(uint64_t seed, long n, signed char* out);

/* ---- allocation-free solve ------------------------------------------------------ */
/* No counterpart in the reference. For callers that cannot allocate device
 * memory (code recording a CUDA graph on another thread, plugins confined to
 * their host application's memory pool, allocator-free latency loops):
 * the reference FP64 CG (as DWF_SOLVER_CG64) for one domain-wall right-hand
 * side, needing no context and calling no cudaMalloc, cudaFree or allocating
 * library routine. The caller passes device pointers it owns: theta_dev
 * (2*Nt*Nx angles), b_dev and x_dev (Ls*Nt*Nx*2 complex<double>; x read as the
 * guess when has_guess), and a cudaStream_t as void* (NULL: the calling
 * thread's per-thread default stream, never the legacy NULL stream). The call
 * returns when the solve is done (it reads its report back). All other
 * buffers live in one static device array that each GPU loading the library
 * holds until exit: lattices up to DWF_NOALLOC_MAX_SITES = Ls*Nt*Nx sites and
 * DWF_NOALLOC_MAX_LINKS = 2*Nt*Nx links; larger ones return DWF_BAD_ARG.
 * params->device selects (and leaves current) the GPU. The first call on a
 * device resolves the array's device address (kept for the process's life,
 * so no use across a cudaDeviceReset), so make that first call before any
 * stream capture. While another thread holds a capture open, that capture
 * must use cudaStreamCaptureModeThreadLocal or ...Relaxed: in global mode
 * CUDA forbids every other thread the synchronous read-back this call makes.
 * Calls share the array: calls whose GPU work overlaps race and must be
 * serialised by the caller. Returns the solve status, or DWF_TIMEOUT when a
 * wait inside the solver ran out; info (host, may be NULL) as dwf_cg reports
 * it, also on DWF_TIMEOUT. */
#define DWF_NOALLOC_MAX_SITES 65536
#define DWF_NOALLOC_MAX_LINKS 32768
int dwf_cg_noalloc(const dwf_params* params, int op, const double* theta_dev, const void* b_dev,
                   void* x_dev, int has_guess, double rtol, int maxiter, void* stream,
                   dwf_solve_info* info);

/* Self test of the bounded grid barrier used by every persistent kernel: one
 * block per SM passes 8 barriers that expect missing_blocks more arrivals than
 * there are blocks. missing_blocks = 0 returns DWF_OK; > 0 makes every wait run
 * into limit_ns and returns DWF_TIMEOUT with the context still usable. */
int dwf_barrier_selftest(dwf_ctx* ctx, int missing_blocks, uint64_t limit_ns);

/* Dslash kernel variant for dwf_apply[_dev]: 0 = one thread per 5-D site,
 * 1 = one thread per 4-D site sweeping the fifth dimension (links and fifth-
 * dimension neighbours kept in registers), 2 = one thread per 5-D site with
 * the x neighbours exchanged by warp shuffles (Nx a multiple of 32; else as
 * 0), 3 = one thread per (s, x) sweeping a chunk of rows in t, the rows
 * streamed through a shared-memory ring by cp.async (Nx a multiple of 32 and
 * Ls <= 16; else as 0), 4 = Wilson contexts only: one thread per four
 * consecutive rows of one column, all loads up front into registers (Nx a
 * multiple of 32 and Nt of 4; else as 0), 5 = as 1 with the x neighbours
 * exchanged by warp shuffles and the next slice's loads issued ahead (Nx a
 * multiple of 32; else as 1), 6 = as 1 with each block's slices (its 32 x 8
 * sites and their halo) brought into a shared-memory ring by 1-D bulk copies
 * completing on mbarriers, every neighbour read from shared memory (Nx a
 * multiple of 32 and Nt of 8; else as 0; chosen only by this call: slower
 * than 5 at the sizes measured; a copy wait that runs past the context's
 * timeout leaves the output incomplete and DWF_TIMEOUT in the device error
 * word that the next solve reports), -1 = autotune (default): the first
 * application per (precision, batch-size bucket) times variants 0-5 with
 * CUDA events and keeps the fastest, variant 3 at its automatic shape and at
 * chunks of 16, 32, 64 and 128 rows with the widest, a half- and a
 * quarter-width block (unless dwf_set_dslash_chunk fixes the chunk). dwf_dslash_variant reports the choice in force for a
 * precision and batch size (-1 if not tuned yet). */
int dwf_set_dslash_variant(dwf_ctx* ctx, int variant);
int dwf_dslash_variant(const dwf_ctx* ctx, int precision, int nrhs);

/* Rows per chunk of variant 3 (0 = automatic: halved from Nt, down to 8,
 * until the grid holds two blocks per resident slot). Clears the autotuner's
 * choices. */
int dwf_set_dslash_chunk(dwf_ctx* ctx, int rows);

/* Kernel of the even-odd Schur solve: -1 automatic (default): one thread-
 * block cluster per right-hand side with its FP32 fields in the cluster's
 * distributed shared memory wherever one right-hand side fits (Nt divisible by
 * the cluster size 8 or 16, Ls/4 in {4, 6}, ~200 KB of fields per CTA) and
 * the device can co-schedule such clusters, else the grid-wide persistent
 * kernel; 0 the grid-wide kernel always. The environment variable
 * DWF_B200_EO_KERNEL=grid makes 0 the default of every context. */
int dwf_set_eo_kernel(dwf_ctx* ctx, int kernel);

/* Per-phase device timers of the even-odd solver kernel (block 0's view, each
 * phase including the grid barrier that ends it): enable (1) allocates and
 * zeroes them, 0 frees them (off by default: no cost). dwf_eo_phase_times
 * returns accumulated ms and counts for the phases 0 hop + M5^-1, 1 M5 - H
 * (|t|^2), 2 alpha reduction, 3 adjoint hop + M5^-1, 4 adjoint combine and
 * x, r update, 5 beta reduction and reliable updates, 6 direction update. */
int dwf_eo_phase_profile(dwf_ctx* ctx, int enable);
int dwf_eo_phase_times(dwf_ctx* ctx, double* ms, uint64_t* counts);

/* ---- device selection ------------------------------------------------------------ */
/* No counterpart in the reference (its executables are CPU programs). Number of
 * CUDA devices visible to this process (DWF_CUDA_ERROR and 0 when none). */
int dwf_device_count(int* count);
/* The next device in turn, modulo ndevices, among the processes of this host
 * that share counter_path (a small text file holding the next index, updated
 * under an exclusive flock): each call takes one index. The drop-in headers
 * call it when DWF_B200_DEVICE=auto, so that the study driver's concurrent
 * cases (scripts/run_three_part_study.py:166-169) run on different GPUs. */
int dwf_round_robin_device(int ndevices, const char* counter_path, int* device);

/* Number of kernels this context has launched so far. */
uint64_t dwf_launch_count(const dwf_ctx* ctx);
/* Accumulated device time (ms) of the persistent solver launches of one kind
 * (0: full-lattice CG kernels, 1: the even-odd Schur solve, either kernel,
 * 2: the even-odd cluster kernel alone), measured with
 * CUDA events on the context stream; *nlaunch (optional) = their count. */
double dwf_solver_kernel_ms(const dwf_ctx* ctx, int kind, uint64_t* nlaunch);
/* Even-odd propagator solves on the cluster kernel (dwf_propagators,
 * dwf_measure and their device forms; no counterpart in the reference) run
 * each chunk's source preparation, solver launch and reconstruction as one
 * CUDA graph, captured on the first call and replayed while the chunk's size,
 * buffers and settings repeat (the 16 most recent are kept per context).
 * Returns the number of replays so far; *cached (optional) = graphs held. */
uint64_t dwf_graph_replays(const dwf_ctx* ctx, int* cached);

/* ---- learned preconditioner (no counterpart in the reference) ------------------ */
/* A gauge-equivariant parallel-transport convolution network N ~ D^-1 of four
 * layers, C0 -> hidden -> hidden -> hidden -> C0 complex channels per 4-D site
 * (C0 = 2 Ls for domain wall, channel 2 s + spin; 2 for Wilson). Layer:
 *   out(y)[o] = sum_{k<9} sum_i W_k[o][i] * T_k(y) in(y + d_k)[i]
 * over the 3x3 stencil offsets d_k = (dt, dx) in the order (0,0) (1,0) (-1,0)
 * (0,1) (0,-1) (1,1) (1,-1) (-1,1) (-1,-1), T_k the U(1) transporter from
 * y + d_k to y with the fermion boundary signs (diagonals: mean of the two
 * two-link paths). No bias or activation, so N is linear and gauge covariant;
 * N^dag runs the layers backwards with W'_k = (W_rev(k))^H. The transported
 * values and the weights are rounded to BF16, the products accumulated in FP32
 * on the tensor cores. Weights: 2 * dwf_lp_weights_size floats (re, im), layer
 * by layer, each [9][cout][cin]. */
int dwf_lp_init(dwf_ctx* ctx, int hidden, uint64_t seed);   /* hidden: 8, 16, 24 or 32; 2 Ls hidden <= 1536, Ls <= 24 */
int dwf_lp_weights_size(const dwf_ctx* ctx, long* n_complex);
int dwf_lp_get_weights(dwf_ctx* ctx, float* w);
int dwf_lp_set_weights(dwf_ctx* ctx, const float* w);
/* Transporters of configuration conf as the kernels use them: [V][9] complex float. */
int dwf_lp_transports(dwf_ctx* ctx, int conf, float* T);
/* out = N in (adjoint != 0: N^dag in) for nrhs FP32 complex fields in the
 * operator layout on the device; rhs_conf as for dwf_cg_batch_dev. */
int dwf_lp_apply_dev(dwf_ctx* ctx, int adjoint, int nrhs, const int* rhs_conf, const void* in_dev,
                     void* out_dev);
/* One layer (adjoint: its adjoint) on FP32 fields in the network layout [V][C]. */
int dwf_lp_layer_dev(dwf_ctx* ctx, int layer, int adjoint, int nrhs, const int* rhs_conf,
                     const void* in_dev, void* out_dev);
/* Training loss (1/B) sum_b |N rho_b - e_b|^2 / |e_b|^2 over npair FP32 pairs
 * (device, operator layout) and its gradient dL/dRe W + i dL/dIm W (host, as
 * the weights; may be NULL). */
int dwf_lp_loss_grad_dev(dwf_ctx* ctx, int npair, const int* pair_conf, const void* rho_dev,
                         const void* e_dev, double* loss, float* grad);
typedef struct
{
    int steps;           /* Adam steps */
    int batch;           /* pairs per step (<= 1024) */
    double lr;           /* Adam learning rate */
    int lr_decay_steps;  /* halve the rate every this many steps (0: constant) */
    int pairs_per_conf;  /* pairs generated per gauge configuration of the context */
    int solver_iters;    /* solver pairs: error of the CG iterate after this many iterations
                            against the converged solution (0: Gaussian errors only) */
    int solver_every;    /* groups of 16 pairs: every solver_every-th is a solver group */
    int solver_maxiter;  /* iteration limit of the converged solve */
    uint64_t seed;
} dwf_lp_train_params;
typedef struct
{
    double loss_first, loss_last;
    int steps, npairs, solver_pairs;
    double seconds_pairs, seconds_train;
} dwf_lp_train_info;
/* Generate pairs (rho = D e) on the context's configurations and train the
 * network with Adam on the GPU; history (host, may be NULL) receives the loss
 * of every step. */
int dwf_lp_train(dwf_ctx* ctx, const dwf_lp_train_params* params, dwf_lp_train_info* info,
                 double* history);
/* Device time of one network application to nrhs Gaussian fields (CUDA
 * events around `reps` back-to-back applications on the context stream) and
 * its arithmetic: 8 * 9 * sum_l cin_l cout_l * V * nrhs real flops. */
int dwf_lp_time_network(dwf_ctx* ctx, int nrhs, int reps, double* ms_per_apply, double* flops_per_apply);
/* Layer kernel: -1 automatic (default: the first DWF_SOLVER_LEARNED solve per
 * batch-size bucket times one network application with each kernel and keeps
 * the faster; the tcgen05 kernel competes only where every layer's shared-
 * memory tile fits; before any solve, the tcgen05 kernel wherever it fits),
 * 0 the mma.sync kernel, 1 the tcgen05 kernel only (DWF_BAD_ARG where it does
 * not fit). */
int dwf_lp_set_variant(dwf_ctx* ctx, int variant);
/* Inner solve: stop at |r| <= inner_tol |r0| or inner_maxiter iterations;
 * at most outer_max defect-correction cycles (defaults 3e-4, 400, 40). */
int dwf_lp_set_solver(dwf_ctx* ctx, double inner_tol, int inner_maxiter, int outer_max);
/* Inner Krylov method of DWF_SOLVER_LEARNED: DWF_LP_GCR (default) is flexible
 * GCR restarted every `restart` iterations (4, 8, 12 or 16; default 4), one
 * network application and one D per iteration: z_k = N r, w_k = D z_k
 * orthogonalised against the cycle's earlier w (classical Gram-Schmidt), the
 * minimal-residual step on r, and the cycle's correction formed from the
 * stored z_k, so N need not be the same operator in every iteration.
 * DWF_LP_BICGSTAB is right-preconditioned BiCGStab (two network applications
 * and two D per iteration; restart ignored). */
enum
{
    DWF_LP_GCR = 0,
    DWF_LP_BICGSTAB = 1
};
int dwf_lp_set_krylov(dwf_ctx* ctx, int method, int restart);


#ifdef __cplusplus
}
#endif


#endif /* DWF_B200_H */
