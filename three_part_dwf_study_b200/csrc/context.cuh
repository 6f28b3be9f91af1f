// Context: device, stream, gauge configurations and solver workspace.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"
#include "solver.cuh"

struct dwf_ctx
{
    int kind = 0;  // 0 domain wall, 1 Wilson
    dwfb::Lat L{};
    double beta = 0.0;
    int device = 0;
    int nsm = 0;
    cudaStream_t stream = nullptr;
    // host-buffer propagator batches: copies on a second stream, overlapped
    // with the solve of the neighbouring chunks (created on first use)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pipe_ev[8] = {};
    uint64_t timeout_ns = 5000000000ull;
    std::string err;
    uint64_t gauge_version = 0;  // bumped whenever the links change
    struct LpNet* lp = nullptr;  // learned preconditioner (dwf_lp_init)
    uint64_t launches = 0;  // kernels launched by this context
    // Dslash kernel variant (-1 autotune, 0-6 as dwf_set_dslash_variant
    // lists them); tuned choices cached per (precision, batch-size bucket),
    // for the t-sweeping kernel with its chunk length and 32-x tiles per block
    // (0: the automatic shape).
    struct DslashChoice
    {
        int variant = 0;
        int tc = 0;
        int g = 0;
    };
    int dslash_variant = -1;
    int dslash_chunk = 0;    // rows per chunk of the t-sweeping Dslash (0 = automatic)
    int sweep_smem_set = 0;  // t-sweeping kernels whose shared-memory limit is raised (bits)
    int l1_pref_set = 0;     // shared-memory-free Dslash kernels asked for the largest L1 (bits)
    int* dslash_err = nullptr;  // device word: DWF_TIMEOUT from a slice-ring Dslash wait (variant 6)
    std::map<int, DslashChoice> dslash_tuned;
    // CUDA events bracketing each persistent solver launch on `stream`
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // device time of solver launches: full lattice, even-odd (either kernel),
    // even-odd cluster kernel alone
    double solver_ms[3] = {0.0, 0.0, 0.0};
    uint64_t solver_launches[3] = {0, 0, 0};

    // gauge configurations
    int nconf = 0;
    int nconf_cap = 0;
    double* theta = nullptr;  // [nconf][2V]
    double2* U64 = nullptr;
    float2* U32 = nullptr;

    // workspace, sized for ws_rhs right-hand sides
    int ws_rhs = 0;
    double2* w_r = nullptr;
    double2* w_p = nullptr;
    double2* w_p2 = nullptr;
    double2* w_t = nullptr;
    double2* w_b = nullptr;  // host-pointer entry points stage b / in here
    double2* w_x = nullptr;  // and x / out here
    float2* w_r32 = nullptr;
    float2* w_p32 = nullptr;
    float2* w_p32b = nullptr;
    float2* w_t32 = nullptr;
    float2* w_e32 = nullptr;
    double* w_part = nullptr;
    size_t w_part_cap = 0;
    double2* w_src = nullptr;  // propagator sources (device staging)
    // dwf_measure's contraction partials, noise-loop sums and Z4 digits
    // (grow-only, like the solver workspace)
    double* m_red = nullptr;
    size_t m_red_cap = 0;
    double2* m_loop = nullptr;
    size_t m_loop_cap = 0;
    signed char* m_z4 = nullptr;
    size_t m_z4_cap = 0;
    int* w_conf = nullptr;
    int* w_active = nullptr;
    int* w_iters = nullptr;
    double* w_relres = nullptr;
    int* w_status = nullptr;
    int* w_ru = nullptr;
    double* w_true = nullptr;
    dwfb::GridBar* bar = nullptr;

    // even-odd workspace (parity fields, allocated on first use)
    int eo_rhs = 0;
    double2* eo_se = nullptr;   // source, even sites
    double2* eo_so = nullptr;   // source, odd sites
    double2* eo_bh = nullptr;   // b_o - H_oe M5^-1 b_e
    double2* eo_rhs_o = nullptr;  // Dhat^dag bhat
    double2* eo_x = nullptr;    // odd solution
    double2* eo_r = nullptr;
    double2* eo_t = nullptr;
    double2* eo_y = nullptr;    // even temporary
    double2* eo_xn = nullptr;
    float2* eo_r32 = nullptr;
    float2* eo_p32 = nullptr;
    float2* eo_t32 = nullptr;
    float2* eo_y32 = nullptr;
    float2* eo_e32 = nullptr;
    unsigned long long* eo_phase = nullptr;  // per-phase timers (dwf_eo_phase_profile)
    int eo_kernel = -1;  // even-odd solver kernel: -1 automatic, 0 grid-wide (dwf_set_eo_kernel)
    // captured even-odd propagator chunks (source preparation, the cluster
    // solver launch, reconstruction), most recent last, replayed when the
    // chunk's size, buffers and settings repeat
    struct GraphEntry
    {
        std::vector<uintptr_t> key;
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0;
    };
    std::vector<GraphEntry> graphs;
    uint64_t graph_replays = 0;

    // HMC workspace (allocated on first use)
    double* h_mom = nullptr;    // [2V]
    double* h_force = nullptr;  // [2V]
    double* h_part = nullptr;   // [2 * kRedBlocks]
    double* h_scal = nullptr;   // [16]
    double2* h_chi = nullptr;   // [fsz]
    double2* h_phi = nullptr;
    double2* h_eta = nullptr;
    double2* h_xi = nullptr;

    long fsz() const { return 2L * L.nsite; }
    long usz() const { return 2L * L.V; }
};

// Device selection, stream, barrier state and events of a new context.
extern "C" int dwfb_ctx_init(dwf_ctx* c, int device);

namespace dwfb {

int ctx_fail(dwf_ctx* c, int code, const std::string& msg);
int ensure_workspace(dwf_ctx* c, int nrhs);
int ensure_part(dwf_ctx* c, size_t n);
// Chunks per right-hand side, sites per chunk and grid size of a persistent
// solver launch over nrhs right-hand sides with `cap` resident blocks.
void choose_units(int nsite, int nrhs, long cap, int* nch, int* ch, int* grid);
// Batched solve on device fields (b, x: nrhs fields of fsz complex doubles).
int solve_batch(dwf_ctx* c, int op, int nrhs, const int* conf_h, const double2* b, double2* x,
                int has_guess, double rtol, int maxiter, int solver, int eigen_rule,
                dwf_solve_info* info);
// FP64 true residual |b - A x| / |b| per right-hand side into host array out.
int true_residual(dwf_ctx* c, int op, int nrhs, const int* conf_d, const double2* b,
                  const double2* x, double* out);
// out = op(in) on device fields, precision 64 or 32.
int apply_dev(dwf_ctx* c, int op, int nrhs, const int* conf_d, int conf0, const void* in,
              void* out, int precision);
// Upload nconf configurations (host or device pointer) and recompute links.
int set_gauge(dwf_ctx* c, int nconf, const double* theta, cudaMemcpyKind kind);
// Even-odd preconditioned solve of D x = src for nrhs sources (device, full
// lattice); returns DWF_BAD_ARG when the lattice does not allow it.
int propagators_eo(dwf_ctx* c, int nrhs, const int* conf_h, const double2* src, double2* x,
                   double tol, int maxiter, std::vector<int>& iters, std::vector<int>& ru);
bool eo_eligible(const dwf_ctx* c);
// Right-hand sides the even-odd cluster solver runs at once on this context's
// lattice and device (its resident clusters), 0 where the cluster path does not apply.
int eo_cluster_wave(dwf_ctx* c);
// Propagator batch: x = (D^dag D)^-1 D^dag src on device fields.
int propagators(dwf_ctx* c, int nrhs, const int* conf_h, const double2* src, double2* x,
                double rtol, int maxiter, int solver, dwf_solve_info* info);

}  // namespace dwfb
