// Allocation-free FP64 CG entry point.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being recorded on another thread, plugins embedded in a host application
// that owns the GPU memory pool and forbids allocations outside it, or
// latency-critical loops that must not hit the allocator. dwf_cg_noalloc
// serves them: the caller passes the gauge angles, the right-hand side and
// the solution buffer (all device memory it already owns), and every other
// buffer the solver needs -- link phases, residual, search directions, the
// operator temporary, partial sums, barrier state and per-solve outputs --
// lives in one file-scope static __device__ array of fixed size that each GPU
// loading this library holds until the process exits.
//
// The array is shared by every call: calls whose GPU work overlaps (on
// different streams, or from different host threads on the same device)
// race on it and must be serialised by the caller. Each call clears what
// must start at zero (the grid-barrier state, and x when no guess is given);
// the rest is written before it is read.
#include <algorithm>
#include <mutex>

#include "context.cuh"
#include "kernels.cuh"

namespace {

using namespace dwfb;

constexpr long kMaxSites = DWF_NOALLOC_MAX_SITES;  // Ls*Nt*Nx 2-spinor sites
constexpr long kMaxLinks = DWF_NOALLOC_MAX_LINKS;  // 2*Nt*Nx link phases
constexpr long kMaxUnits = 4096;                   // (rhs, chunk) units of the solver
constexpr long kPartDoubles = kMaxUnits * 2 > (kMaxSites + 4095) / 4096 * 2
                                  ? kMaxUnits * 2
                                  : (kMaxSites + 4095) / 4096 * 2;

// Byte offsets of the scratch regions (each 256-byte aligned).
constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }
constexpr size_t kField = align256(size_t(kMaxSites) * 2 * sizeof(double2));
constexpr size_t kOffR = 0;
constexpr size_t kOffP = kOffR + kField;
constexpr size_t kOffP2 = kOffP + kField;
constexpr size_t kOffT = kOffP2 + kField;
constexpr size_t kOffU64 = kOffT + kField;
constexpr size_t kOffU32 = kOffU64 + align256(size_t(kMaxLinks) * sizeof(double2));
constexpr size_t kOffPart = kOffU32 + align256(size_t(kMaxLinks) * sizeof(float2));
constexpr size_t kOffBar = kOffPart + align256(size_t(kPartDoubles) * sizeof(double));
constexpr size_t kOffOut = kOffBar + align256(sizeof(GridBar));
constexpr size_t kOutBytes = 4 * sizeof(int) + 2 * sizeof(double);
constexpr size_t kScratchBytes = kOffOut + align256(kOutBytes);

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_base[kMaxDevices] = {};

// Device address of g_scratch on `dev` (must be current). In host code the
// name g_scratch is only a host-side stand-in, never a device address. The
// address is resolved on the first call per device and kept for the life of
// the process: a cudaDeviceReset of that device (which unloads the module)
// leaves it stale, so the entry point must not be used across a device reset.
int scratch_base(int dev, unsigned char** base)
{
    if (dev < 0 || dev >= kMaxDevices)
        return DWF_BAD_ARG;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_base[dev])
    {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p)
            return DWF_CUDA_ERROR;
        g_base[dev] = p;
    }
    *base = static_cast<unsigned char*>(g_base[dev]);
    return DWF_OK;
}

}  // namespace

extern "C" int dwf_cg_noalloc(const dwf_params* p, int op, const double* theta_dev,
                              const void* b_dev, void* x_dev, int has_guess, double rtol,
                              int maxiter, void* stream_ptr, dwf_solve_info* info)
{
    if (!p || !theta_dev || !b_dev || !x_dev || (op != DWF_OP_DDDAG && op != DWF_OP_DDAGD) ||
        maxiter < 0 || !(rtol >= 0.0) || p->Nt < 1 || p->Nx < 1 || p->Ls < 1)
        return DWF_BAD_ARG;
    const long V = long(p->Nt) * p->Nx;
    const long nsite = V * p->Ls;
    if (nsite > kMaxSites || 2 * V > kMaxLinks)
        return DWF_BAD_ARG;  // beyond DWF_NOALLOC_MAX_SITES / DWF_NOALLOC_MAX_LINKS
    if (cudaSetDevice(p->device) != cudaSuccess)
        return DWF_CUDA_ERROR;
    unsigned char* base = nullptr;
    int st = scratch_base(p->device, &base);
    if (st)
        return st;
    // NULL selects the calling thread's per-thread default stream, never the
    // legacy NULL stream: work on the legacy stream would implicitly
    // synchronise with (and so invalidate) a capture that another thread holds
    // open on a blocking stream.
    cudaStream_t stream =
        stream_ptr ? static_cast<cudaStream_t>(stream_ptr) : cudaStreamPerThread;
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess)
        return DWF_CUDA_ERROR;

    Lat L{};
    L.Nt = p->Nt;
    L.Nx = p->Nx;
    L.Ls = p->Ls;
    L.V = int(V);
    L.nsite = int(nsite);
    L.diag = 3.0 - p->M5;
    L.mf = p->mf;
    L.bct = -1.0;
    L.bcx = 1.0;
    L.fifth = 1;

    double2* r = reinterpret_cast<double2*>(base + kOffR);
    double2* pp = reinterpret_cast<double2*>(base + kOffP);
    double2* p2 = reinterpret_cast<double2*>(base + kOffP2);
    double2* t = reinterpret_cast<double2*>(base + kOffT);
    double2* U64 = reinterpret_cast<double2*>(base + kOffU64);
    float2* U32 = reinterpret_cast<float2*>(base + kOffU32);
    double* part = reinterpret_cast<double*>(base + kOffPart);
    GridBar* bar = reinterpret_cast<GridBar*>(base + kOffBar);
    int* o_iters = reinterpret_cast<int*>(base + kOffOut);
    int* o_status = o_iters + 1;
    int* o_ru = o_iters + 2;
    int* o_conf = o_iters + 3;  // rhs_conf[0] = 0
    double* o_relres = reinterpret_cast<double*>(base + kOffOut + 4 * sizeof(int));
    double* o_true = o_relres + 1;

    const long fs = 2 * nsite;
    links_kernel<<<int(std::min<long>((2 * V + 255) / 256, 8L * nsm)), 256, 0, stream>>>(
        theta_dev, 2 * V, U64, U32);
    if (cudaMemsetAsync(bar, 0, sizeof(GridBar), stream) != cudaSuccess ||
        cudaMemsetAsync(o_conf, 0, sizeof(int), stream) != cudaSuccess)
        return DWF_CUDA_ERROR;
    if (!has_guess && cudaMemsetAsync(x_dev, 0, fs * sizeof(double2), stream) != cudaSuccess)
        return DWF_CUDA_ERROR;

    SolveDesc d{};
    d.L = L;
    d.dag_first = (op == DWF_OP_DDDAG) ? 1 : 0;
    d.nrhs = 1;
    d.fsz = fs;
    d.rhs_conf = o_conf;
    d.U64 = U64;
    d.U32 = U32;
    d.usz = 2 * V;
    d.b = static_cast<const double2*>(b_dev);
    d.x = static_cast<double2*>(x_dev);
    d.r = r;
    d.p = pp;
    d.p2 = p2;
    d.t = t;
    d.rtol = rtol;
    d.maxiter = maxiter;
    d.has_guess = has_guess;
    d.out_iters = o_iters;
    d.out_relres = o_relres;
    d.out_status = o_status;
    d.out_ru = o_ru;
    d.bar = bar;
    d.timeout_ns = 5000000000ull;

    const void* fn = reinterpret_cast<const void*>(&cg64_kernel<true, 2>);
    const size_t smem = solver_smem_bytes(1);
    int bps = 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, 256, smem) != cudaSuccess ||
        bps < 1)
        return DWF_CUDA_ERROR;
    const long cap = long(bps) * nsm;
    // the same work units as the context-based solver (identical reduction order)
    int grid = 0;
    choose_units(int(nsite), 1, std::min<long>(cap, kMaxUnits), &d.nch, &d.ch, &grid);
    d.part = part;
    d.expected_blocks = unsigned(grid);
    void* args[] = {&d};
    if (cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, smem, stream) != cudaSuccess)
        return DWF_CUDA_ERROR;

    // FP64 true residual |b - A x| / |b| with the scratch temporary t
    const dim3 g1(int(std::min<long>((nsite + 255) / 256, 4L * nsm)), 1);
    if (d.dag_first)
        dirac_kernel<true, double><<<g1, 256, 0, stream>>>(L, d.x, t, fs, U64, 2 * V, o_conf, 0);
    else
        dirac_kernel<false, double><<<g1, 256, 0, stream>>>(L, d.x, t, fs, U64, 2 * V, o_conf, 0);
    const int rch = 4096;
    const int rnch = int((nsite + rch - 1) / rch);
    if (d.dag_first)
        residual_partials_kernel<false><<<dim3(rnch, 1), 256, 0, stream>>>(L, t, d.b, fs, U64, 2 * V, o_conf, rnch, rch, part);
    else
        residual_partials_kernel<true><<<dim3(rnch, 1), 256, 0, stream>>>(L, t, d.b, fs, U64, 2 * V, o_conf, rnch, rch, part);
    residual_finish_kernel<<<1, 256, 0, stream>>>(part, 1, rnch, o_true);
    if (cudaGetLastError() != cudaSuccess)
        return DWF_CUDA_ERROR;

    int hi[4];
    double hd[2];
    GridBar hb{};
    if (cudaMemcpyAsync(hi, o_iters, sizeof(hi), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaMemcpyAsync(hd, o_relres, sizeof(hd), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaMemcpyAsync(&hb, bar, sizeof(hb), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return DWF_CUDA_ERROR;
    // a barrier error (a wait that ran out) outranks the solver's own status
    const int status = hb.err != 0 ? hb.err : hi[1];
    if (info)
    {
        info->iterations = hi[0];
        info->status = status;
        info->converged = status == DWF_OK ? 1 : 0;
        info->solver = DWF_SOLVER_CG64;
        info->relres = hd[0];
        info->true_relres = hd[1];
        info->reliable_updates = 0;
        info->fallback = 0;
        info->dirac_relres = 0.0;
        info->schur_iterations = 0;
    }
    return status;
}
