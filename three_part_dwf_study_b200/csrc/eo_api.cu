// Host side of the even-odd preconditioned propagator solve.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "context.cuh"
#include "eo.cuh"

using namespace dwfb;

#define CK(call)                                                                        \
    do                                                                                  \
    {                                                                                   \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ctx_fail(c, DWF_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

namespace dwfb {

__global__ void eo_pack_kernel(Lat L, EoGeo g, const double2* full, double2* ev, double2* od,
                               long nrhs);
__global__ void eo_unpack_kernel(Lat L, EoGeo g, const double2* ev, const double2* od,
                                 double2* full, long nrhs);
template <bool DAG>
__global__ void eo_hopinv_kernel(Lat L, EoGeo g, const double2* in, const double2* src,
                                 double sgn, double2* out, const double2* U, long usz,
                                 const int* conf, long nrhs);
template <bool DAG>
__global__ void eo_combine_kernel(Lat L, EoGeo g, const double2* a, const double2* m,
                                  const double2* y, double2* out, const double2* U, long usz,
                                  const int* conf, long nrhs);
__global__ void cg_eo_mixed_kernel(EoDesc e);
int launch_eo_cluster(dwf_ctx* c, EoDesc& e, bool* launched, bool dry, int* wave = nullptr);

// DWF_B200_EO_KERNEL=grid keeps every even-odd solve on the grid-wide kernel
// (cg_eo_mixed_kernel); by default the cluster kernel (eo_cluster.cu) takes
// the batches whose right-hand side fits a cluster's shared memory.
bool eo_cluster_enabled()
{
    static const bool on = [] {
        const char* v = std::getenv("DWF_B200_EO_KERNEL");
        return !(v && std::strcmp(v, "grid") == 0);
    }();
    return on;
}

bool eo_eligible(const dwf_ctx* c)
{
    return c->kind == 0 && c->L.Nt % 2 == 0 && c->L.Nx % 2 == 0 && c->L.diag >= 1.0;
}

int eo_cluster_wave(dwf_ctx* c)
{
    if (!eo_eligible(c) || c->eo_kernel == 0 || !eo_cluster_enabled())
        return 0;
    EoDesc e{};
    e.d.nrhs = 1;
    e.d.delta = 0.1;
    bool ok = false;
    int wave = 0;
    if (launch_eo_cluster(c, e, &ok, true, &wave) != DWF_OK || !ok)
        return 0;
    return wave;
}

namespace {

int ensure_eo(dwf_ctx* c, int nrhs)
{
    if (nrhs <= c->eo_rhs)
        return DWF_OK;
    CK(cudaStreamSynchronize(c->stream));
    void** bufs64[] = {reinterpret_cast<void**>(&c->eo_se), reinterpret_cast<void**>(&c->eo_so),
                       reinterpret_cast<void**>(&c->eo_bh), reinterpret_cast<void**>(&c->eo_rhs_o),
                       reinterpret_cast<void**>(&c->eo_x), reinterpret_cast<void**>(&c->eo_r),
                       reinterpret_cast<void**>(&c->eo_t), reinterpret_cast<void**>(&c->eo_y),
                       reinterpret_cast<void**>(&c->eo_xn)};
    void** bufs32[] = {reinterpret_cast<void**>(&c->eo_r32), reinterpret_cast<void**>(&c->eo_p32),
                       reinterpret_cast<void**>(&c->eo_t32), reinterpret_cast<void**>(&c->eo_y32),
                       reinterpret_cast<void**>(&c->eo_e32)};
    const size_t fh = size_t(nrhs) * c->L.nsite;  // complex entries of one parity field (2 * nsite / 2)
    c->eo_rhs = 0;
    for (void** b : bufs64)
    {
        if (*b)
            cudaFree(*b);
        *b = nullptr;
        CK(cudaMalloc(b, fh * sizeof(double2)));
    }
    for (void** b : bufs32)
    {
        if (*b)
            cudaFree(*b);
        *b = nullptr;
        CK(cudaMalloc(b, fh * sizeof(float2)));
    }
    c->eo_rhs = nrhs;
    return DWF_OK;
}

constexpr size_t kGraphCache = 16;

// Run `body` (stream work only) through a CUDA graph cached under `key`:
// replay it if present, else capture it on the context stream (thread-local
// mode) and launch the instantiated graph. If capture or instantiation fails,
// `body` runs again directly. The cache keeps the kGraphCache most recent
// graphs.
template <typename F>
int run_graph(dwf_ctx* c, const std::vector<uintptr_t>& key, F body)
{
    for (size_t i = 0; i < c->graphs.size(); ++i)
        if (c->graphs[i].key == key)
        {
            dwf_ctx::GraphEntry g = c->graphs[i];
            c->graphs.erase(c->graphs.begin() + long(i));
            c->graphs.push_back(g);
            CK(cudaGraphLaunch(g.exec, c->stream));
            c->launches += g.launches;
            c->graph_replays += 1;
            return DWF_OK;
        }
    // errors pending from earlier calls are the caller's; capture only from a clean state
    if (cudaPeekAtLastError() != cudaSuccess)
        return body();
    const uint64_t l0 = c->launches;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int st = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (st == DWF_OK && e == cudaSuccess && graph &&
        cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess)
    {
        cudaGraphDestroy(graph);
        if (c->graphs.size() >= kGraphCache)
        {
            cudaGraphExecDestroy(c->graphs.front().exec);
            c->graphs.erase(c->graphs.begin());
        }
        c->graphs.push_back({key, exec, c->launches - l0});
        CK(cudaGraphLaunch(exec, c->stream));
        return DWF_OK;
    }
    if (graph)
        cudaGraphDestroy(graph);
    cudaGetLastError();
    c->launches = l0;
    return body();
}

}  // namespace

int propagators_eo(dwf_ctx* c, int nrhs, const int* conf_h, const double2* src, double2* x,
                   double tol, int maxiter, std::vector<int>& iters, std::vector<int>& ru)
{
    if (!eo_eligible(c))
        return ctx_fail(c, DWF_BAD_ARG, "even-odd solve needs even Nt, Nx and 3 - M5 >= 1");
    constexpr int kMaxRhs = 2048;
    iters.assign(nrhs, 0);
    ru.assign(nrhs, 0);
    EoGeo g{c->L.Nx / 2, c->L.V / 2};
    const long fh = long(g.Vh) * c->L.Ls * 2;  // complex entries per parity field
    const long fs = c->fsz();
    for (int k0 = 0; k0 < nrhs; k0 += kMaxRhs)
    {
        const int n = std::min(kMaxRhs, nrhs - k0);
        int st = ensure_workspace(c, n);
        if (st || (st = ensure_eo(c, n)))
            return st;
        std::vector<int> conf(n, 0);
        if (conf_h)
            std::copy(conf_h + k0, conf_h + k0 + n, conf.begin());
        CK(cudaMemcpyAsync(c->w_conf, conf.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        const int nb = std::max(1, 8 * c->nsm);
        const long usz = c->usz();
        // b_e, b_o; bhat = b_o - H_oe M5^-1 b_e; rhs = Dhat^dag bhat; x_o = 0
        auto prepare = [&]() -> int {
            eo_pack_kernel<<<nb, 256, 0, c->stream>>>(c->L, g, src + k0 * fs, c->eo_se, c->eo_so, n);
            eo_hopinv_kernel<false><<<nb, 256, 0, c->stream>>>(c->L, g, nullptr, c->eo_se, 1.0, c->eo_y, c->U64, usz, c->w_conf, n);
            eo_combine_kernel<false><<<nb, 256, 0, c->stream>>>(c->L, g, c->eo_so, nullptr, c->eo_y, c->eo_bh, c->U64, usz, c->w_conf, n);
            eo_hopinv_kernel<true><<<nb, 256, 0, c->stream>>>(c->L, g, c->eo_bh, nullptr, 1.0, c->eo_y, c->U64, usz, c->w_conf, n);
            eo_combine_kernel<true><<<nb, 256, 0, c->stream>>>(c->L, g, nullptr, c->eo_bh, c->eo_y, c->eo_rhs_o, c->U64, usz, c->w_conf, n);
            CK(cudaGetLastError());
            c->launches += 5;
            CK(cudaMemsetAsync(c->eo_x, 0, size_t(n) * fh * sizeof(double2), c->stream));
            return DWF_OK;
        };
        // x_e = M5^-1 (b_e - H_eo x_o); x = (x_e, x_o)
        auto reconstruct = [&]() -> int {
            eo_hopinv_kernel<false><<<nb, 256, 0, c->stream>>>(c->L, g, c->eo_x, c->eo_se, -1.0, c->eo_y, c->U64, usz, c->w_conf, n);
            eo_unpack_kernel<<<nb, 256, 0, c->stream>>>(c->L, g, c->eo_y, c->eo_x, x + k0 * fs, n);
            CK(cudaGetLastError());
            c->launches += 2;
            return DWF_OK;
        };

        EoDesc e{};
        SolveDesc& d = e.d;
        d.L = c->L;
        d.L.nsite = g.Vh * c->L.Ls;  // persistent sweeps run over odd 5-D sites
        d.nrhs = n;
        d.fsz = fh;
        d.rhs_conf = c->w_conf;
        d.U64 = c->U64;
        d.U32 = c->U32;
        d.usz = usz;
        d.b = c->eo_rhs_o;
        d.x = c->eo_x;
        d.r = c->eo_r;
        d.t = c->eo_t;
        d.r32 = c->eo_r32;
        d.p32 = c->eo_p32;
        d.t32 = c->eo_t32;
        d.e32 = c->eo_e32;
        d.rtol = tol;
        d.maxiter = maxiter;
        d.delta = 0.1;
        d.stall_limit = 3;
        d.ru_period = d.nrhs > 1 ? kRuPeriod : 1;   // batching pays only across right-hand sides
        d.out_iters = c->w_iters;
        d.out_relres = c->w_relres;
        d.out_status = c->w_status;
        d.out_ru = c->w_ru;
        d.bar = c->bar;
        d.timeout_ns = c->timeout_ns;
        e.g = g;
        e.y64 = c->eo_y;
        e.y32 = c->eo_y32;
        e.xn64 = c->eo_xn;
        e.phase_ns = c->eo_phase;

        bool clustered = false;
        if (c->eo_kernel != 0 && eo_cluster_enabled())
        {
            st = launch_eo_cluster(c, e, &clustered, true);
            if (st != DWF_OK && st != DWF_BAD_ARG)
                return st;
        }
        if (clustered)
        {
            // preparation, the cluster solver and the reconstruction as one
            // graph, replayed while the chunk's buffers and settings repeat
            const std::vector<uintptr_t> key = {
                uintptr_t(n), uintptr_t(src + k0 * fs), uintptr_t(x + k0 * fs), uintptr_t(c->w_conf),
                uintptr_t(c->U64), uintptr_t(c->U32), uintptr_t(c->eo_se), uintptr_t(c->eo_so),
                uintptr_t(c->eo_bh), uintptr_t(c->eo_rhs_o), uintptr_t(c->eo_x), uintptr_t(c->eo_r),
                uintptr_t(c->eo_t), uintptr_t(c->eo_y), uintptr_t(c->eo_xn), uintptr_t(c->eo_r32),
                uintptr_t(c->eo_p32), uintptr_t(c->eo_t32), uintptr_t(c->eo_y32), uintptr_t(c->eo_e32),
                uintptr_t(c->w_iters), uintptr_t(c->w_relres), uintptr_t(c->w_status), uintptr_t(c->w_ru),
                uintptr_t(c->eo_phase), uintptr_t(c->bar), uintptr_t(maxiter), uintptr_t(c->timeout_ns),
                uintptr_t(std::llround(std::log2(tol) * 1e6)), uintptr_t(d.ru_period)};
            st = run_graph(c, key, [&]() -> int {
                int s2 = prepare();
                if (s2)
                    return s2;
                // external records: event nodes of the graph, not capture markers
                CK(cudaEventRecordWithFlags(c->ev0, c->stream, cudaEventRecordExternal));
                bool l = false;
                s2 = launch_eo_cluster(c, e, &l, false);
                if (s2 || !l)
                    return s2 ? s2 : ctx_fail(c, DWF_CUDA_ERROR, "even-odd cluster solver: launch failed");
                CK(cudaEventRecordWithFlags(c->ev1, c->stream, cudaEventRecordExternal));
                c->launches += 1;
                return reconstruct();
            });
            if (st)
                return st;
            std::vector<int> it(n), r(n);
            CK(cudaMemcpyAsync(it.data(), c->w_iters, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaMemcpyAsync(r.data(), c->w_ru, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
            c->solver_ms[1] += ms;
            c->solver_launches[1] += 1;
            c->solver_ms[2] += ms;
            c->solver_launches[2] += 1;
            for (int k = 0; k < n; ++k)
            {
                iters[k0 + k] = it[k];
                ru[k0 + k] = r[k];
            }
            continue;
        }
        st = prepare();
        if (st)
            return st;

        const void* fn = reinterpret_cast<const void*>(&cg_eo_mixed_kernel);
        // the FP32 hop + M5^-1 phases keep each thread's Ls slices in shared
        // memory when that costs no resident blocks (registers bound them)
        const size_t smem_base = solver_smem_bytes(n);
        const size_t smem_z = ((smem_base + 15) & ~size_t(15)) + size_t(256) * c->L.Ls * sizeof(float4);
        int bps_base = 0, bps_z = 0;
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_base)));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_base, fn, 256, smem_base));
        if (smem_z <= size_t(200 * 1024))
        {
            CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_z)));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_z, fn, 256, smem_z));
        }
        e.zsmem = (bps_z >= bps_base && bps_z > 0) ? 1 : 0;
        const size_t smem = e.zsmem ? smem_z : smem_base;
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int bps = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, 256, smem));
        if (bps < 1)
            return ctx_fail(c, DWF_CUDA_ERROR, "even-odd solver kernel cannot be resident");
        const long cap = long(bps) * c->nsm;
        int grid = 0;
        choose_units(d.L.nsite, n, cap, &d.nch, &d.ch, &grid);
        // 4-D even sites: at most one unit per block, so the phase ends after one
        // unit's time (a unit count just above the grid made a few blocks take
        // two units while the rest waited at the barrier), at least 32 sites each
        e.nch4 = int(std::max<long>(1, std::min<long>(g.Vh / 32, grid / n)));
        e.ch4 = (g.Vh + e.nch4 - 1) / e.nch4;
        e.nch4 = (g.Vh + e.ch4 - 1) / e.ch4;
        st = ensure_part(c, size_t(n) * d.nch * 2);
        if (st)
            return st;
        d.part = c->w_part;
        d.expected_blocks = unsigned(grid);
        CK(cudaMemsetAsync(c->bar, 0, sizeof(GridBar), c->stream));
        void* args[] = {&e};
        CK(cudaEventRecord(c->ev0, c->stream));
        CK(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, smem, c->stream));
        CK(cudaEventRecord(c->ev1, c->stream));
        c->launches += 1;
        std::vector<int> it(n), r(n);
        GridBar hb{};
        CK(cudaMemcpyAsync(it.data(), c->w_iters, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(r.data(), c->w_ru, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(&hb, c->bar, sizeof(GridBar), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->solver_ms[1] += ms;
        c->solver_launches[1] += 1;
        if (hb.err != 0)
            return ctx_fail(c, hb.err, "even-odd solver: grid barrier wait ran out");
        for (int k = 0; k < n; ++k)
        {
            iters[k0 + k] = it[k];
            ru[k0 + k] = r[k];
        }
        st = reconstruct();
        if (st)
            return st;
    }
    return DWF_OK;
}

}  // namespace dwfb

extern "C" {

int dwf_eo_phase_profile(dwf_ctx* c, int enable)
{
    if (!c)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    if (enable && !c->eo_phase)
        CK(cudaMalloc(&c->eo_phase, 16 * sizeof(unsigned long long)));
    if (!enable && c->eo_phase)
    {
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(c->eo_phase);
        c->eo_phase = nullptr;
    }
    if (c->eo_phase)
        CK(cudaMemsetAsync(c->eo_phase, 0, 16 * sizeof(unsigned long long), c->stream));
    return DWF_OK;
}

int dwf_set_eo_kernel(dwf_ctx* c, int kernel)
{
    if (!c || kernel < -1 || kernel > 0)
        return DWF_BAD_ARG;
    c->eo_kernel = kernel;
    return DWF_OK;
}

int dwf_eo_phase_times(dwf_ctx* c, double* ms, uint64_t* counts)
{
    if (!c || !c->eo_phase || !ms)
        return DWF_BAD_ARG;
    unsigned long long h[16];
    CK(cudaMemcpyAsync(h, c->eo_phase, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 8; ++k)
    {
        ms[k] = double(h[k]) * 1e-6;
        if (counts)
            counts[k] = h[8 + k];
    }
    return DWF_OK;
}

}  // extern "C"
