// C ABI: contexts, gauge upload, operator application and the batched solver.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "context.cuh"
#include "learned.cuh"
#include "kernels.cuh"

using namespace dwfb;

// The even-odd path's Schur solve stops at this multiple of the requested
// tolerance (on its own normal equation); the full-lattice mixed solve that
// follows, warm-started from it, enforces the reference's rule on D^dag D.
// Warm-started batched mixed solves run FP64 reliable updates every
// DWFB_RU_PERIOD_WARM iterations (a check that starts next to the solution
// should not wait a full period). Measured on the 64x64x16, 28-source
// propagator set with the grid-wide Schur kernel and an unconditional
// full-lattice solve (solves/s, warm period / factor): 16 / 0.3 -> 737,
// 16 / 3 -> 789-795, 16 / 10 -> 699, 8 / 5 -> 780, 4 / 2.5 -> 818,
// 4 / 3 -> 829, 4 / 4 -> 788, 4 / 6 -> 735, 2 / 3 -> 828, 2 / 4 -> 786.
// The full-lattice solve now runs only when the FP64 residual of the full
// normal equation misses the tolerance after the Schur solve; with the
// cluster Schur kernel (GPU-HMC configuration, factor: solves/s): 3 -> 1252,
// 1 -> 1311, 0.5 -> 1267, 0.3 -> 1265; on three configurations of the chain
// 1 -> 1311 / 1339 / 1329, 0.85 -> 1306 / 1329 / 1314, 0.7 -> 1293 / 1324 / 1293.
// At 0.7 - 3 the check still misses by a little and the full-lattice mixed
// solve adds at most 4 iterations per source (about 0.6 ms per 28-source batch).
// The full-lattice solve in FP64 (DWFB_EO_POLISH_SOLVER) checks the true residual
// every iteration where the warm-started mixed one waits for its first reliable
// update: 2-3 iterations, and a looser Schur stop then pays (three
// configurations, solves/s): mixed, factor 1 -> 1313 / 1346 / 1334; FP64, 1 ->
// 1331 / 1365 / 1354; 1.5 -> 1368 / 1387 / 1364; 2 -> 1385 / 1403 / 1377; 3 ->
// 1404 / 1401 / 1393 (up to 5 iterations); 4 -> 1127 / 1150 / 1142 (up to 67:
// past about 3x the full-lattice solve has to remove the Schur solution's low
// modes). 2 keeps a margin below that edge. Where the grid-wide Schur kernel
// runs (right-hand sides too large for a cluster) the same pair cost the
// finite-volume study at 64x96x16 (1792 sources) 20 % (451.5 against 561.9
// solves/s; 64x80x16: 719.6 against 706.5), so that path keeps factor 1 and
// the mixed check solve.
#ifndef DWFB_EO_SCHUR_TOL
#define DWFB_EO_SCHUR_TOL 2.0       // cluster Schur kernel
#endif
#ifndef DWFB_EO_POLISH_SOLVER
#define DWFB_EO_POLISH_SOLVER DWF_SOLVER_CG64
#endif
#ifndef DWFB_EO_SCHUR_TOL_GRID
#define DWFB_EO_SCHUR_TOL_GRID 1.0  // grid-wide Schur kernel
#endif
#ifndef DWFB_EO_POLISH_SOLVER_GRID
#define DWFB_EO_POLISH_SOLVER_GRID DWF_SOLVER_MIXED
#endif
#ifndef DWFB_PIPE_CHUNKS
// Chunks of a host-buffer even-odd cluster batch (1 to 4). At 64x64x16 with 28
// sources (four waves), page-locked buffers: 1 chunk 29.0 ms per batch, 2 chunks
// 28.5, 4 chunks 29.1 (a chunk ends with its slowest wave; one launch lets each
// cluster run its right-hand sides back to back); the device-buffer call 26.9.
#define DWFB_PIPE_CHUNKS 2
#endif
#ifndef DWFB_RU_PERIOD_WARM
#define DWFB_RU_PERIOD_WARM 4
#endif

#define CK(call)                                                                        \
    do                                                                                  \
    {                                                                                   \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ctx_fail(c, DWF_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

namespace dwfb {

int ctx_fail(dwf_ctx* c, int code, const std::string& msg)
{
    if (c)
        c->err = msg;
    return code;
}

namespace {

template <typename T>
int grow(dwf_ctx* c, T*& p, size_t n)
{
    if (p)
        cudaFree(p);
    p = nullptr;
    if (n == 0)
        return DWF_OK;
    CK(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)));
    return DWF_OK;
}

}  // namespace

int ensure_workspace(dwf_ctx* c, int nrhs)
{
    if (nrhs <= c->ws_rhs)
        return DWF_OK;
    CK(cudaStreamSynchronize(c->stream));
    const size_t f = size_t(nrhs) * c->fsz();
    int st;
    if ((st = grow(c, c->w_r, f)) || (st = grow(c, c->w_p, f)) || (st = grow(c, c->w_p2, f)) ||
        (st = grow(c, c->w_t, f)) || (st = grow(c, c->w_p32b, f)) ||
        (st = grow(c, c->w_b, f)) || (st = grow(c, c->w_x, f)) || (st = grow(c, c->w_r32, f)) ||
        (st = grow(c, c->w_p32, f)) || (st = grow(c, c->w_t32, f)) ||
        (st = grow(c, c->w_e32, f)) || (st = grow(c, c->w_src, f)) ||
        (st = grow(c, c->w_conf, size_t(nrhs))) ||
        (st = grow(c, c->w_active, size_t(nrhs))) || (st = grow(c, c->w_iters, size_t(nrhs))) ||
        (st = grow(c, c->w_relres, size_t(nrhs))) || (st = grow(c, c->w_status, size_t(nrhs))) ||
        (st = grow(c, c->w_ru, size_t(nrhs))) || (st = grow(c, c->w_true, size_t(nrhs))))
    {
        c->ws_rhs = 0;
        return st;
    }
    c->ws_rhs = nrhs;
    return DWF_OK;
}

void choose_units(int nsite, int nrhs, long cap, int* nch_out, int* ch_out, int* grid_out)
{
    // Work units = (right-hand side, chunk). Pick the chunk count that fills
    // the resident blocks in whole waves (every block gets the same number of
    // units, up to one), preferring fewer, larger chunks.
    int best_nch = 1;
    long best_waves = 1;
    double best_eff = -1.0;
    for (int nch = 1; nch <= 4096; ++nch)
    {
        const long ch_try = (nsite + nch - 1) / nch;
        if (nch > 1 && ch_try < 128)
            break;
        const long u = long(nrhs) * nch;
        const long waves = (u + cap - 1) / cap;
        const double eff = double(u) / double(waves * cap);
        if (eff > best_eff + 0.02)
        {
            best_eff = eff;
            best_nch = nch;
            best_waves = waves;
        }
        if (eff >= 0.95)
            break;
    }
    const int ch = (nsite + best_nch - 1) / best_nch;
    const int nch = (nsite + ch - 1) / ch;
    const long units = long(nrhs) * nch;
    *nch_out = nch;
    *ch_out = ch;
    *grid_out = int(std::min<long>(cap, (units + best_waves - 1) / best_waves));
}

int ensure_part(dwf_ctx* c, size_t n)
{
    if (n <= c->w_part_cap)
        return DWF_OK;
    CK(cudaStreamSynchronize(c->stream));
    const int st = grow(c, c->w_part, n);
    c->w_part_cap = st ? 0 : n;
    return st;
}

#ifndef DWFB_DIRAC_BLOCKS_PER_SM
#define DWFB_DIRAC_BLOCKS_PER_SM 4  // grid cap of the site kernel (0: one site per thread)
#endif

namespace {

// One application of D (dag = false) or D^dag with the chosen kernel variant.
// The t-sweeping kernel needs whole 32-lane rows and a block of all Ls slices.
bool sweep_ok(const Lat& L) { return L.Nx % 32 == 0 && 32 * L.Ls <= 512; }
bool tile_ok(const Lat& L) { return L.Nx % 32 == 0 && L.Nt % kRingT == 0; }
bool wilson_rows_ok(const Lat& L)
{
    return L.Ls == 1 && !L.fifth && L.Nx % 32 == 0 && L.Nt % kWilsonRows == 0;
}

struct SweepShape
{
    int g;   // 32-x tiles per block
    int tc;  // rows per chunk
};

// Blocks of up to 512 threads (G tiles of 32 x 32 Ls threads); the chunk
// length is the context's setting, else halved from Nt (down to 8 rows) until
// the grid holds at least two blocks per resident slot (1024 resident threads
// per SM, as the kernel's launch bounds allow), so the tail of the launch
// stays short.
// Largest dynamic shared memory of one block (the sweep's ring must fit).
constexpr size_t kSweepSmemMax = 227 * 1024;

SweepShape sweep_shape(const dwf_ctx* c, int nrhs, int resident_threads, int ring_rows, size_t csize)
{
    const Lat& L = c->L;
    int g = 1;
    while (32 * L.Ls * g * 2 <= 512 && (L.Nx / 32) % (g * 2) == 0 &&
           ring_rows * sweep_slot_bytes(L.Ls, g * 2, csize) <= kSweepSmemMax)
        g *= 2;
    const long nxt = L.Nx / (32 * g);
    int tc = c->dslash_chunk > 0 ? std::min(c->dslash_chunk, L.Nt) : L.Nt;
    if (c->dslash_chunk <= 0)
    {
        const long slots = long(c->nsm) * std::max(1, resident_threads / (32 * L.Ls * g));
        while (tc > 8 && nxt * ((L.Nt + tc - 1) / tc) * nrhs < 2 * slots)
            tc = (tc + 1) / 2;
    }
    return {g, tc};
}

using DslashChoice = dwf_ctx::DslashChoice;

// The t-sweeping kernel's compile-time shape per precision.
template <typename R>
struct SweepCfg
{
    static constexpr int NPG = sizeof(R) == 8 ? kSweepGroups64 : kSweepGroups32;
    static constexpr int RPS = sizeof(R) == 8 ? kSweepRows64 : kSweepRows32;
    static constexpr int S = sweep_ring_rows(NPG, RPS);
    // resident threads per SM as the kernel's launch bounds allow
    static constexpr int resident = (sizeof(R) == 8 && RPS == 2) ? 512 : 1024;
};

template <typename R>
SweepShape auto_sweep_shape(const dwf_ctx* c, int nrhs)
{
    return sweep_shape(c, nrhs, SweepCfg<R>::resident, SweepCfg<R>::S, sizeof(cplx<R>));
}

// The kernels that use no shared memory lean on L1 for their neighbour reuse
// (and the column kernel for its prefetched slices). Without a preference the
// driver may keep a small-L1 split chosen for a preceding shared-memory-heavy
// kernel (the t sweep, the network layers), so ask once per kernel for the
// largest L1; a refusal only leaves the default split.
template <typename K>
void prefer_l1(dwf_ctx* c, int bit, K kern)
{
    if (c->l1_pref_set & (1 << bit))
        return;
    // a refusal is not an error of the launch that follows: clear it, unless an
    // earlier error is pending for the caller's check
    const bool clean = cudaPeekAtLastError() == cudaSuccess;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             int(cudaSharedmemCarveoutMaxL1)) != cudaSuccess &&
        clean)
        cudaGetLastError();
    c->l1_pref_set |= 1 << bit;
}

template <typename R>
void launch_dirac(dwf_ctx* c, DslashChoice ch, bool dag, int nrhs, const int* conf_d, int conf0,
                  const cplx<R>* in, cplx<R>* out, const cplx<R>* U)
{
    const long fs = c->fsz();
    const int variant = ch.variant;
    if (variant == 3 && sweep_ok(c->L))
    {
        constexpr int NPG = SweepCfg<R>::NPG, RPS = SweepCfg<R>::RPS, S = SweepCfg<R>::S;
        const SweepShape sh = ch.tc > 0 ? SweepShape{ch.g, ch.tc} : auto_sweep_shape<R>(c, nrhs);
        const dim3 grid(c->L.Nx / (32 * sh.g), (c->L.Nt + sh.tc - 1) / sh.tc, nrhs);
        const dim3 block(32, c->L.Ls, sh.g);
        const size_t smem = S * sweep_slot_bytes(c->L.Ls, sh.g, sizeof(cplx<R>));
        auto kern = dag ? dirac_sweep_kernel<true, R, NPG, RPS> : dirac_sweep_kernel<false, R, NPG, RPS>;
        const int bit = (dag ? 1 : 0) + (sizeof(R) == 8 ? 2 : 0);
        if (!(c->sweep_smem_set & (1 << bit)))
        {
            // the largest ring this context's lattice can ask for (G = 1 .. 512 / (32 Ls));
            // a failure here leaves the launch below to fail, which the caller's
            // cudaGetLastError check reports
            size_t most = 0;
            for (int g = 1; 32 * c->L.Ls * g <= 512; g *= 2)
            {
                const size_t b = S * sweep_slot_bytes(c->L.Ls, g, sizeof(cplx<R>));
                if (b <= kSweepSmemMax)
                    most = std::max(most, b);
            }
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(most)) ==
                cudaSuccess)
                c->sweep_smem_set |= 1 << bit;
        }
        kern<<<grid, block, smem, c->stream>>>(c->L, in, out, fs, U, c->usz(), conf_d, conf0, sh.tc);
    }
    else if (variant == 4 && wilson_rows_ok(c->L))
    {
        constexpr int by = 8;
        const dim3 grid(c->L.Nx / 32, (c->L.Nt / kWilsonRows + by - 1) / by, nrhs);
        const dim3 block(32, by);
        if (dag)
            wilson_rows_kernel<true, R, kWilsonRows><<<grid, block, 0, c->stream>>>(c->L, in, out, fs, U, c->usz(), conf_d, conf0);
        else
            wilson_rows_kernel<false, R, kWilsonRows><<<grid, block, 0, c->stream>>>(c->L, in, out, fs, U, c->usz(), conf_d, conf0);
    }
    else if (variant == 5 && c->L.Nx % 32 == 0)
    {
        const dim3 grid(c->L.Nx / 32, (c->L.Nt + 7) / 8, nrhs);
        auto kern = dag ? dirac_colx_kernel<true, R> : dirac_colx_kernel<false, R>;
        prefer_l1(c, 0 + (dag ? 1 : 0) + (sizeof(R) == 8 ? 2 : 0), kern);
        kern<<<grid, 256, 0, c->stream>>>(c->L, in, out, fs, U, c->usz(), conf_d, conf0);
    }
    else if (variant == 6 && tile_ok(c->L) && c->dslash_err)
    {
        const dim3 grid(c->L.Nx / 32, c->L.Nt / kRingT, nrhs);
        auto kern = dag ? dirac_tile_kernel<true, R> : dirac_tile_kernel<false, R>;
        const int bit = 8 + (dag ? 1 : 0) + (sizeof(R) == 8 ? 2 : 0);
        if (!(c->sweep_smem_set & (1 << bit)))
        {
            // several blocks' rings per SM need the largest shared-memory split;
            // a refusal only leaves fewer blocks resident
            const bool clean = cudaPeekAtLastError() == cudaSuccess;
            if ((cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      int(cudaSharedmemCarveoutMaxShared)) != cudaSuccess ||
                 cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(tile_smem_bytes(2 * sizeof(cplx<R>)))) != cudaSuccess) &&
                clean)
                cudaGetLastError();
            c->sweep_smem_set |= 1 << bit;
        }
        kern<<<grid, 256, tile_smem_bytes(2 * sizeof(cplx<R>)), c->stream>>>(
            c->L, in, out, fs, U, c->usz(), conf_d, conf0, c->dslash_err, c->timeout_ns);
    }
    else if (variant == 1 || variant == 5)
    {
        const dim3 grid((c->L.Nx + 31) / 32, (c->L.Nt + 7) / 8, nrhs);
        auto kern = dag ? dirac_col_kernel<true, R> : dirac_col_kernel<false, R>;
        prefer_l1(c, 4 + (dag ? 1 : 0) + (sizeof(R) == 8 ? 2 : 0), kern);
        kern<<<grid, 256, 0, c->stream>>>(c->L, in, out, fs, U, c->usz(), conf_d, conf0);
    }
    else
    {
        const int nb = (c->L.nsite + 255) / 256;
        const int bx = DWFB_DIRAC_BLOCKS_PER_SM > 0
                           ? std::min(nb, std::max(1, DWFB_DIRAC_BLOCKS_PER_SM * c->nsm))
                           : nb;
        const dim3 grid(bx, nrhs);
        const int b = (dag ? 1 : 0) + (sizeof(R) == 8 ? 2 : 0);
        if (variant == 2 && c->L.Nx % 32 == 0)
        {
            auto kern = dag ? dirac_warp_kernel<true, R> : dirac_warp_kernel<false, R>;
            prefer_l1(c, 8 + b, kern);
            kern<<<grid, 256, 0, c->stream>>>(c->L, in, out, fs, U, c->usz(), conf_d, conf0);
        }
        else
        {
            auto kern = dag ? dirac_kernel<true, R> : dirac_kernel<false, R>;
            prefer_l1(c, 12 + b, kern);
            kern<<<grid, 256, 0, c->stream>>>(c->L, in, out, fs, U, c->usz(), conf_d, conf0);
        }
    }
    c->launches += 1;
}

// Autotuner: time the variants (two applications each, CUDA events on the
// context stream) for this precision and batch-size bucket, keep the fastest:
// 0 one thread per 5-D site, 1 one thread per 4-D column, 2 one thread per 5-D
// site with warp-shuffled x neighbours (Nx a multiple of 32), 3 one thread per
// (s, x) sweeping a chunk of rows in t (Nx a multiple of 32, Ls <= 16), 4 (Wilson
// only) one thread per kWilsonRows rows of one column from registers, 5 one
// thread per 4-D column with warp-shuffled x neighbours (Nx a multiple of 32); the
// slice-ring kernel (6) is not a candidate (slower than 5 wherever measured). Unless
// the context fixes the chunk length, the t sweep is timed at its automatic
// shape and at chunks of 16, 32, 64 and 128 rows with the widest block and
// with a half and a quarter of its 32-x tiles: long chunks amortise the ring's
// start-up, narrower blocks keep enough of them to fill the SMs.
template <typename R>
DslashChoice pick_variant(dwf_ctx* c, int nrhs, const int* conf_d, int conf0, const cplx<R>* in,
                          cplx<R>* out, const cplx<R>* U)
{
    if (c->dslash_variant >= 0)
        return {c->dslash_variant, 0, 0};
    int bucket = 0;
    while ((1 << bucket) < nrhs && bucket < 20)
        ++bucket;
    const int key = (sizeof(R) == 8 ? 100 : 0) + bucket;
    auto it = c->dslash_tuned.find(key);
    if (it != c->dslash_tuned.end())
        return it->second;
    std::vector<DslashChoice> cand;
    for (int v = 0; v < 6; ++v)
    {
        if (((v == 2 || v == 5) && c->L.Nx % 32 != 0) || (v == 3 && !sweep_ok(c->L)) ||
            (v == 4 && !wilson_rows_ok(c->L)))
            continue;
        cand.push_back({v, 0, 0});
        if (v == 3 && c->dslash_chunk <= 0)
        {
            const SweepShape a = auto_sweep_shape<R>(c, nrhs);
            for (int g = a.g; g >= 1 && g * 4 >= a.g; g /= 2)
                for (int tc : {16, 32, 64, 128})
                    if (tc <= c->L.Nt && !(g == a.g && tc == a.tc))
                        cand.push_back({3, tc, g});
        }
    }
    // an error already pending belongs to the caller: tune only from a clean state
    if (cudaPeekAtLastError() != cudaSuccess)
        return cand.front();
    float best = 1e30f;
    bool any = false;
    DslashChoice choice = cand.front();
    for (const DslashChoice& ch : cand)
    {
        launch_dirac<R>(c, ch, false, nrhs, conf_d, conf0, in, out, U);  // warm-up
        cudaEventRecord(c->ev0, c->stream);
        for (int k = 0; k < 2; ++k)
            launch_dirac<R>(c, ch, false, nrhs, conf_d, conf0, in, out, U);
        cudaEventRecord(c->ev1, c->stream);
        cudaEventSynchronize(c->ev1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        // a candidate that failed to launch did no work: drop it rather than time it
        if (cudaGetLastError() != cudaSuccess)
        {
            // an error that reading does not clear is sticky: the context is
            // lost, so stop launching into it
            if (cudaPeekAtLastError() != cudaSuccess)
                break;
            continue;
        }
        any = true;
        if (ms < best)
        {
            best = ms;
            choice = ch;
        }
    }
    // cache only a choice that ran; with none, the caller's own launch reports
    // the error and the next call tunes again
    if (any)
        c->dslash_tuned[key] = choice;
    return choice;
}

}  // namespace

int apply_dev(dwf_ctx* c, int op, int nrhs, const int* conf_d, int conf0, const void* in,
              void* out, int precision)
{
    if (nrhs < 1 || nrhs > 65535 || op < 0 || op > 3 || (precision != 64 && precision != 32))
        return ctx_fail(c, DWF_BAD_ARG, "apply: bad op, nrhs or precision");
    if (conf0 < 0 || conf0 >= c->nconf)
        return ctx_fail(c, DWF_BAD_ARG, "apply: configuration index out of range (set_gauge first)");
    // the kernels move a spin pair (FP32) or a complex number (FP64) per 16-byte access
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
        return ctx_fail(c, DWF_BAD_ARG, "apply: fields must start on a 16-byte boundary");
    const bool two = (op == DWF_OP_DDDAG || op == DWF_OP_DDAGD);
    if (two)
    {
        const int st = ensure_workspace(c, nrhs);
        if (st)
            return st;
    }
    // first (or only) operator: D for D, D^dag D; D^dag for D^dag, D D^dag
    const bool dag1 = (op == DWF_OP_DDAG || op == DWF_OP_DDDAG);
    if (precision == 64)
    {
        const double2* src = static_cast<const double2*>(in);
        double2* mid = two ? c->w_t : static_cast<double2*>(out);
        const DslashChoice v = pick_variant<double>(c, nrhs, conf_d, conf0, src, mid, c->U64);
        launch_dirac<double>(c, v, dag1, nrhs, conf_d, conf0, src, mid, c->U64);
        if (two)
            launch_dirac<double>(c, v, !dag1, nrhs, conf_d, conf0, mid, static_cast<double2*>(out), c->U64);
    }
    else
    {
        const float2* src = static_cast<const float2*>(in);
        float2* mid = two ? c->w_t32 : static_cast<float2*>(out);
        const DslashChoice v = pick_variant<float>(c, nrhs, conf_d, conf0, src, mid, c->U32);
        launch_dirac<float>(c, v, dag1, nrhs, conf_d, conf0, src, mid, c->U32);
        if (two)
            launch_dirac<float>(c, v, !dag1, nrhs, conf_d, conf0, mid, static_cast<float2*>(out), c->U32);
    }
    CK(cudaGetLastError());
    return DWF_OK;
}

int true_residual(dwf_ctx* c, int op, int nrhs, const int* conf_d, const double2* b,
                  const double2* x, double* out)
{
    // t = D1 x
    const bool dag1 = (op == DWF_OP_DDDAG);
    const long fs = c->fsz();
    const dim3 block(256);
    const dim3 grid(std::min((c->L.nsite + 255) / 256, std::max(1, 4 * c->nsm)), nrhs);
    if (dag1)
        dirac_kernel<true, double><<<grid, block, 0, c->stream>>>(c->L, x, c->w_t, fs, c->U64, c->usz(), conf_d, 0);
    else
        dirac_kernel<false, double><<<grid, block, 0, c->stream>>>(c->L, x, c->w_t, fs, c->U64, c->usz(), conf_d, 0);
    const int ch = 4096;
    const int nch = (c->L.nsite + ch - 1) / ch;
    int st = ensure_part(c, size_t(nrhs) * nch * 2);
    if (st)
        return st;
    const dim3 g2(nch, nrhs);
    if (dag1)
        residual_partials_kernel<false><<<g2, block, 0, c->stream>>>(c->L, c->w_t, b, fs, c->U64, c->usz(), conf_d, nch, ch, c->w_part);
    else
        residual_partials_kernel<true><<<g2, block, 0, c->stream>>>(c->L, c->w_t, b, fs, c->U64, c->usz(), conf_d, nch, ch, c->w_part);
    residual_finish_kernel<<<(nrhs + 7) / 8, 256, 0, c->stream>>>(c->w_part, nrhs, nch, c->w_true);
    CK(cudaGetLastError());
    c->launches += 3;
    CK(cudaMemcpyAsync(out, c->w_true, nrhs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

namespace {

constexpr int kSolverThreads = 256;
constexpr int kMaxRhsPerLaunch = 2048;

// One persistent launch over nrhs <= kMaxRhsPerLaunch right-hand sides.
int launch_solver(dwf_ctx* c, bool mixed, int op, int nrhs, const double2* b, double2* x,
                  int has_guess, const int* active_d, double rtol, int maxiter, int eigen_rule,
                  std::vector<int>& iters, std::vector<double>& relres, std::vector<int>& status,
                  std::vector<int>& ru)
{
    SolveDesc d{};
    d.L = c->L;
    d.dag_first = (op == DWF_OP_DDDAG) ? 1 : 0;
    d.nrhs = nrhs;
    d.fsz = c->fsz();
    d.rhs_conf = c->w_conf;
    d.U64 = c->U64;
    d.U32 = c->U32;
    d.usz = c->usz();
    d.b = b;
    d.x = x;
    d.r = c->w_r;
    d.p = c->w_p;
    d.p2 = c->w_p2;
    d.t = c->w_t;
    d.r32 = c->w_r32;
    d.p32 = c->w_p32;
    d.p32b = c->w_p32b;
    d.t32 = c->w_t32;
    d.e32 = c->w_e32;
    d.rtol = rtol;
    d.maxiter = maxiter;
    d.has_guess = has_guess;
    d.active_in = active_d;
    d.eigen_rule = eigen_rule;
    d.delta = 0.1;
    d.stall_limit = 3;
    // batching reliable updates pays when right-hand sides would otherwise
    // trigger them on different iterations; a single one only waits longer
    d.ru_period = (mixed && nrhs > 1) ? (has_guess ? DWFB_RU_PERIOD_WARM : kRuPeriod) : 1;
    d.out_iters = c->w_iters;
    d.out_relres = c->w_relres;
    d.out_status = c->w_status;
    d.out_ru = c->w_ru;
    d.bar = c->bar;
    d.timeout_ns = c->timeout_ns;

    // single right-hand side: fused two-barrier iteration; batches: three barriers
    const bool single = nrhs == 1;
    const void* fn = mixed ? (single ? reinterpret_cast<const void*>(&cg_mixed_kernel<true, 2>)
                                     : reinterpret_cast<const void*>(&cg_mixed_kernel<false, 3>))
                           : (single ? reinterpret_cast<const void*>(&cg64_kernel<true, 2>)
                                     : reinterpret_cast<const void*>(&cg64_kernel<false, 3>));
    const size_t smem = solver_smem_bytes(nrhs);
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int bps = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, kSolverThreads, smem));
    if (bps < 1)
        return ctx_fail(c, DWF_CUDA_ERROR, "solver kernel cannot be resident");
    const int cap = bps * c->nsm;
    int grid_blocks = 0;
    choose_units(c->L.nsite, nrhs, cap, &d.nch, &d.ch, &grid_blocks);
    const long units = long(nrhs) * d.nch;
    int st = ensure_part(c, size_t(units) * 2);
    if (st)
        return st;
    d.part = c->w_part;
    const int grid = grid_blocks;
    d.expected_blocks = unsigned(grid);
    CK(cudaMemsetAsync(c->bar, 0, sizeof(GridBar), c->stream));
    void* args[] = {&d};
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kSolverThreads), args, smem, c->stream));
    CK(cudaEventRecord(c->ev1, c->stream));
    c->launches += 1;
    GridBar hb{};
    iters.resize(nrhs);
    relres.resize(nrhs);
    status.resize(nrhs);
    ru.resize(nrhs);
    CK(cudaMemcpyAsync(iters.data(), c->w_iters, nrhs * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(relres.data(), c->w_relres, nrhs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(status.data(), c->w_status, nrhs * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(ru.data(), c->w_ru, nrhs * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&hb, c->bar, sizeof(GridBar), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->solver_ms[0] += ms;
    c->solver_launches[0] += 1;
    if (hb.err != 0)
        return ctx_fail(c, hb.err, hb.err == DWF_TIMEOUT ? "persistent solver: a grid barrier wait ran out"
                                                          : "persistent solver: device error");
    return DWF_OK;
}

}  // namespace

int solve_batch(dwf_ctx* c, int op, int nrhs, const int* conf_h, const double2* b, double2* x,
                int has_guess, double rtol, int maxiter, int solver, int eigen_rule,
                dwf_solve_info* info)
{
    if (op != DWF_OP_DDDAG && op != DWF_OP_DDAGD)
        return ctx_fail(c, DWF_BAD_ARG, "cg: op must be DWF_OP_DDDAG or DWF_OP_DDAGD");
    if (nrhs < 1 || maxiter < 0 || !(rtol >= 0.0) ||
        (solver != DWF_SOLVER_CG64 && solver != DWF_SOLVER_MIXED && solver != DWF_SOLVER_EO_MIXED))
        return ctx_fail(c, DWF_BAD_ARG, "cg: bad nrhs, maxiter, rtol or solver");
    if (solver == DWF_SOLVER_EO_MIXED)
        solver = DWF_SOLVER_MIXED;  // a general right-hand side has no source to precondition
    if (c->nconf < 1)
        return ctx_fail(c, DWF_BAD_ARG, "cg: no gauge configuration (set_gauge first)");
    for (int k = 0; conf_h && k < nrhs; ++k)
        if (conf_h[k] < 0 || conf_h[k] >= c->nconf)
            return ctx_fail(c, DWF_BAD_ARG, "cg: configuration index out of range");
    const long fs = c->fsz();
    for (int k0 = 0; k0 < nrhs; k0 += kMaxRhsPerLaunch)
    {
        const int n = std::min(kMaxRhsPerLaunch, nrhs - k0);
        int st = ensure_workspace(c, n);
        if (st)
            return st;
        std::vector<int> conf(n, 0);
        if (conf_h)
            std::copy(conf_h + k0, conf_h + k0 + n, conf.begin());
        CK(cudaMemcpyAsync(c->w_conf, conf.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        const double2* bk = b + k0 * fs;
        double2* xk = x + k0 * fs;
        if (!has_guess)
            CK(cudaMemsetAsync(xk, 0, size_t(n) * fs * sizeof(double2), c->stream));
        std::vector<int> iters, status, ru;
        std::vector<double> relres;
        const bool mixed = (solver == DWF_SOLVER_MIXED);
        st = launch_solver(c, mixed, op, n, bk, xk, has_guess, nullptr, rtol, maxiter, eigen_rule,
                           iters, relres, status, ru);
        if (st)
            return st;
        std::vector<int> fallback(n, 0);
        int nfb = 0;
        if (mixed)
        {
            for (int k = 0; k < n; ++k)
                if (status[k] != DWF_OK)
                {
                    fallback[k] = 1;
                    ++nfb;
                }
            if (nfb)
            {
                // plain FP64 CG from the mixed iterate for every right-hand side that stalled
                CK(cudaMemcpyAsync(c->w_active, fallback.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
                std::vector<int> it2, st2, ru2;
                std::vector<double> rr2;
                st = launch_solver(c, false, op, n, bk, xk, 1, c->w_active, rtol, maxiter,
                                   eigen_rule, it2, rr2, st2, ru2);
                if (st)
                    return st;
                for (int k = 0; k < n; ++k)
                    if (fallback[k])
                    {
                        iters[k] += it2[k];
                        relres[k] = rr2[k];
                        status[k] = st2[k];
                    }
            }
        }
        std::vector<double> tr(n);
        st = true_residual(c, op, n, c->w_conf, bk, xk, tr.data());
        if (st)
            return st;
        for (int k = 0; info && k < n; ++k)
        {
            dwf_solve_info& I = info[k0 + k];
            I.iterations = iters[k];
            I.status = status[k];
            I.converged = status[k] == DWF_OK ? 1 : 0;
            I.solver = solver;
            I.relres = relres[k];
            I.true_relres = tr[k];
            I.reliable_updates = ru[k];
            I.fallback = fallback[k];
            I.dirac_relres = 0.0;
            I.schur_iterations = 0;
            if (!std::isfinite(tr[k]) && I.status == DWF_OK)
                I.status = DWF_NONFINITE;
        }
    }
    return DWF_OK;
}

int dirac_residual(dwf_ctx* c, int nrhs, const int* conf_d, const double2* src,
                   const double2* x, double* out)
{
    // |src - D x|^2 and |src|^2 per right-hand side
    const int ch = 4096;
    const int nch = (c->L.nsite + ch - 1) / ch;
    int st = ensure_part(c, size_t(nrhs) * nch * 2);
    if (st)
        return st;
    residual_partials_kernel<false><<<dim3(nch, nrhs), 256, 0, c->stream>>>(
        c->L, x, src, c->fsz(), c->U64, c->usz(), conf_d, nch, ch, c->w_part);
    residual_finish_kernel<<<(nrhs + 7) / 8, 256, 0, c->stream>>>(c->w_part, nrhs, nch, c->w_true);
    CK(cudaGetLastError());
    c->launches += 2;
    CK(cudaMemcpyAsync(out, c->w_true, nrhs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int propagators(dwf_ctx* c, int nrhs, const int* conf_h, const double2* src, double2* x,
                double rtol, int maxiter, int solver, dwf_solve_info* info)
{
    if (nrhs < 1)
        return ctx_fail(c, DWF_BAD_ARG, "propagators: nrhs < 1");
    if (c->nconf < 1)
        return ctx_fail(c, DWF_BAD_ARG, "propagators: no gauge configuration (set_gauge first)");
    for (int k = 0; conf_h && k < nrhs; ++k)
        if (conf_h[k] < 0 || conf_h[k] >= c->nconf)
            return ctx_fail(c, DWF_BAD_ARG, "propagators: configuration index out of range");
    int st = ensure_workspace(c, nrhs);
    if (st)
        return st;
    const long fs = c->fsz();
    if (solver == DWF_SOLVER_LEARNED)
    {
        for (int k0 = 0; k0 < nrhs; k0 += 65535)
        {
            const int n = std::min(65535, nrhs - k0);
            st = lp_solve(c, n, conf_h ? conf_h + k0 : nullptr, src + k0 * fs, x + k0 * fs, rtol,
                          maxiter, info ? info + k0 : nullptr);
            if (st)
                return st;
        }
    }
    else
    {
    // rhs = D^dag src, per configuration, into w_b (chunks of up to 65535 fields)
    std::vector<int> conf(nrhs, 0);
    if (conf_h)
        std::copy(conf_h, conf_h + nrhs, conf.begin());
    for (int k0 = 0; k0 < nrhs; k0 += 65535)
    {
        const int n = std::min(65535, nrhs - k0);
        CK(cudaMemcpyAsync(c->w_conf, conf.data() + k0, n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        st = apply_dev(c, DWF_OP_DDAG, n, c->w_conf, 0, src + k0 * fs, c->w_b + k0 * fs, 64);
        if (st)
            return st;
    }
    if (solver == DWF_SOLVER_EO_MIXED && eo_eligible(c))
    {
        // Even-odd Schur solve of D x = src as the starting point, then the
        // full-lattice solve on D^dag D from it: the reference's
        // stopping rule |D^dag D x - D^dag src| <= rtol |D^dag src| decides.
        std::vector<int> eo_it, eo_ru;
        const bool clustered = eo_cluster_wave(c) > 0;
        const double schur_tol = (clustered ? DWFB_EO_SCHUR_TOL : DWFB_EO_SCHUR_TOL_GRID) * rtol;
        st = propagators_eo(c, nrhs, conf_h, src, x, schur_tol, maxiter, eo_it, eo_ru);
        if (st)
            return st;
        // The reference's rule on the full normal equation, in FP64: where every
        // right-hand side meets it already, the full-lattice solve is skipped.
        std::vector<double> tr(nrhs);
        bool all_ok = true;
        for (int k0 = 0; k0 < nrhs; k0 += 65535)
        {
            const int n = std::min(65535, nrhs - k0);
            CK(cudaMemcpyAsync(c->w_conf, conf.data() + k0, n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
            st = true_residual(c, DWF_OP_DDAGD, n, c->w_conf, c->w_b + k0 * fs, x + k0 * fs, tr.data() + k0);
            if (st)
                return st;
        }
        for (int k = 0; k < nrhs; ++k)
            all_ok = all_ok && std::isfinite(tr[k]) && tr[k] <= rtol;
        if (all_ok)
        {
            for (int k = 0; info && k < nrhs; ++k)
            {
                dwf_solve_info& I = info[k];
                I = dwf_solve_info{};
                I.iterations = eo_it[k];
                I.converged = 1;
                I.status = DWF_OK;
                I.relres = tr[k];
                I.true_relres = tr[k];
                I.reliable_updates = eo_ru[k];
                I.schur_iterations = eo_it[k];
                I.solver = DWF_SOLVER_EO_MIXED;
            }
        }
        else
        {
            // the full-lattice solve on D^dag D from the even-odd solution
            st = solve_batch(c, DWF_OP_DDAGD, nrhs, conf_h, c->w_b, x, 1, rtol, maxiter,
                             clustered ? DWFB_EO_POLISH_SOLVER : DWFB_EO_POLISH_SOLVER_GRID, 0, info);
            if (st)
                return st;
            for (int k = 0; info && k < nrhs; ++k)
            {
                info[k].iterations += eo_it[k];
                info[k].schur_iterations = eo_it[k];
                info[k].reliable_updates += eo_ru[k];
                info[k].solver = DWF_SOLVER_EO_MIXED;
            }
        }
    }
    else
    {
        st = solve_batch(c, DWF_OP_DDAGD, nrhs, conf_h, c->w_b, x, 0, rtol, maxiter,
                         solver == DWF_SOLVER_EO_MIXED ? DWF_SOLVER_MIXED : solver,
                         c->kind == 1 ? 1 : 0, info);
        if (st)
            return st;
    }
    }
    std::vector<int> conf(nrhs, 0);
    if (conf_h)
        std::copy(conf_h, conf_h + nrhs, conf.begin());
    for (int k0 = 0; k0 < nrhs; k0 += 65535)
    {
        const int n = std::min(65535, nrhs - k0);
        CK(cudaMemcpyAsync(c->w_conf, conf.data() + k0, n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        std::vector<double> dr(n);
        st = dirac_residual(c, n, c->w_conf, src + k0 * fs, x + k0 * fs, dr.data());
        if (st)
            return st;
        for (int k = 0; info && k < n; ++k)
            info[k0 + k].dirac_relres = dr[k];
    }
    return DWF_OK;
}

}  // namespace dwfb

// ---------------------------------------------------------------------------
// exported entry points
// ---------------------------------------------------------------------------
extern "C" {

const char* dwf_status_string(int s)
{
    switch (s)
    {
    case DWF_OK: return "ok";
    case DWF_NOT_CONVERGED: return "not converged";
    case DWF_ZERO_DENOM: return "CG encountered a zero denominator";
    case DWF_NONFINITE: return "non-finite value";
    case DWF_CUDA_ERROR: return "CUDA error";
    case DWF_TIMEOUT: return "device wait timed out";
    case DWF_BAD_ARG: return "bad argument";
    default: return "unknown status";
    }
}

int dwfb_ctx_init(dwf_ctx* c, int device)
{
    c->device = device;
    CK(cudaSetDevice(device));
    CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&c->bar, sizeof(GridBar)));
    CK(cudaMemset(c->bar, 0, sizeof(GridBar)));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    return DWF_OK;
}

int dwf_ctx_create(const dwf_params* p, dwf_ctx** out)
{
    if (!p || !out)
        return DWF_BAD_ARG;
    *out = nullptr;
    if (p->Nt < 1 || p->Nx < 1 || p->Ls < 1 || long(p->Nt) * p->Nx * p->Ls > (1L << 30))
        return DWF_BAD_ARG;
    dwf_ctx* c = new dwf_ctx();
    c->kind = 0;
    c->L.Nt = p->Nt;
    c->L.Nx = p->Nx;
    c->L.Ls = p->Ls;
    c->L.V = p->Nt * p->Nx;
    c->L.nsite = p->Ls * c->L.V;
    c->L.diag = 3.0 - p->M5;
    c->L.mf = p->mf;
    c->L.bct = -1.0;
    c->L.bcx = 1.0;
    c->L.fifth = 1;
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

int dwf_ctx_destroy(dwf_ctx* c)
{
    if (!c)
        return DWF_OK;
    cudaSetDevice(c->device);
    if (c->stream)
        cudaStreamSynchronize(c->stream);
    lp_destroy(c);
    void* bufs[] = {c->h_mom, c->h_force, c->h_part, c->h_scal, c->h_chi, c->h_phi, c->h_eta,
                    c->h_xi, c->theta, c->U64, c->U32, c->w_r, c->w_p, c->w_p2, c->w_p32b, c->w_t, c->w_b, c->w_x,
                    c->w_r32, c->w_p32, c->w_t32, c->w_e32, c->w_src, c->w_part, c->w_conf, c->w_active,
                    c->w_iters, c->w_relres, c->w_status, c->w_ru, c->w_true, c->bar, c->dslash_err,
                    c->eo_se, c->eo_so, c->eo_bh, c->eo_rhs_o, c->eo_x, c->eo_r, c->eo_t, c->eo_y,
                    c->eo_xn, c->eo_r32, c->eo_p32, c->eo_t32, c->eo_y32, c->eo_e32,
                    c->eo_phase, c->m_red, c->m_loop, c->m_z4};
    for (void* b : bufs)
        if (b)
            cudaFree(b);
    for (auto& g : c->graphs)
        if (g.exec)
            cudaGraphExecDestroy(g.exec);
    if (c->ev0)
        cudaEventDestroy(c->ev0);
    if (c->ev1)
        cudaEventDestroy(c->ev1);
    for (cudaEvent_t ev : c->pipe_ev)
        if (ev)
            cudaEventDestroy(ev);
    if (c->copy_stream)
    {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->stream)
        cudaStreamDestroy(c->stream);
    delete c;
    return DWF_OK;
}

const char* dwf_last_error(const dwf_ctx* c) { return c ? c->err.c_str() : ""; }

int dwf_set_wait_limit(dwf_ctx* c, uint64_t ns)
{
    if (!c || ns == 0)
        return DWF_BAD_ARG;
    c->timeout_ns = ns;
    return DWF_OK;
}

int dwf_sync(dwf_ctx* c)
{
    if (!c)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

void* dwf_stream(dwf_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

}  // extern "C"

namespace dwfb {
int set_gauge(dwf_ctx* c, int nconf, const double* theta, cudaMemcpyKind kind)
{
    if (!c || nconf < 1 || !theta)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    const long n = long(nconf) * c->usz();
    if (nconf > c->nconf_cap)
    {
        CK(cudaStreamSynchronize(c->stream));
        if (c->theta) cudaFree(c->theta);
        if (c->U64) cudaFree(c->U64);
        if (c->U32) cudaFree(c->U32);
        c->theta = nullptr;
        c->U64 = nullptr;
        c->U32 = nullptr;
        c->nconf_cap = 0;
        CK(cudaMalloc(&c->theta, n * sizeof(double)));
        CK(cudaMalloc(&c->U64, n * sizeof(double2)));
        CK(cudaMalloc(&c->U32, n * sizeof(float2)));
        c->nconf_cap = nconf;
    }
    CK(cudaMemcpyAsync(c->theta, theta, n * sizeof(double), kind, c->stream));
    const int grid = int(std::min<long>((n + 255) / 256, 8L * c->nsm));
    links_kernel<<<grid, 256, 0, c->stream>>>(c->theta, n, c->U64, c->U32);
    CK(cudaGetLastError());
    c->launches += 1;
    CK(cudaStreamSynchronize(c->stream));
    c->nconf = nconf;
    c->gauge_version += 1;
    return DWF_OK;
}

// dwf_propagators in chunks of `chunk` right-hand sides (at most four); the
// workspace is already sized for all nrhs, so no chunk reallocates the
// buffers the copies use. Whatever fails, both streams are drained before
// returning, so that no copy touches the caller's buffers afterwards.
int propagators_pipelined(dwf_ctx* c, int nrhs, const int* rhs_conf, const double* src, double* x,
                          double rtol, int maxiter, int solver, dwf_solve_info* info, int chunk)
{
    const long fs = c->fsz();
    const int nchunk = (nrhs + chunk - 1) / chunk;
    if (nchunk > 4)
        return ctx_fail(c, DWF_BAD_ARG, "propagators: more than four chunks");
    if (!c->copy_stream)
        CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& ev : c->pipe_ev)
        if (!ev)
            CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    const size_t field = size_t(fs) * sizeof(double2);
    int st = DWF_OK;
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < nchunk && ce == cudaSuccess; ++k)
    {
        const int k0 = k * chunk, n = std::min(chunk, nrhs - k0);
        ce = cudaMemcpyAsync(c->w_src + k0 * fs, src + 2 * k0 * fs, n * field, cudaMemcpyHostToDevice,
                             c->copy_stream);
        if (ce == cudaSuccess)
            ce = cudaEventRecord(c->pipe_ev[k], c->copy_stream);
    }
    for (int k = 0; k < nchunk && ce == cudaSuccess && st == DWF_OK; ++k)
    {
        const int k0 = k * chunk, n = std::min(chunk, nrhs - k0);
        ce = cudaStreamWaitEvent(c->stream, c->pipe_ev[k], 0);
        if (ce != cudaSuccess)
            break;
        st = propagators(c, n, rhs_conf ? rhs_conf + k0 : nullptr, c->w_src + k0 * fs, c->w_x + k0 * fs,
                         rtol, maxiter, solver, info ? info + k0 : nullptr);
        if (st)
            break;
        ce = cudaEventRecord(c->pipe_ev[4 + k], c->stream);
        if (ce == cudaSuccess)
            ce = cudaStreamWaitEvent(c->copy_stream, c->pipe_ev[4 + k], 0);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(x + 2 * k0 * fs, c->w_x + k0 * fs, n * field, cudaMemcpyDeviceToHost,
                                 c->copy_stream);
    }
    const cudaError_t e1 = cudaStreamSynchronize(c->copy_stream);
    const cudaError_t e2 = cudaStreamSynchronize(c->stream);
    if (st)
        return st;
    CK(ce);
    CK(e1);
    CK(e2);
    return DWF_OK;
}

}  // namespace dwfb

extern "C" {

int dwf_set_gauge(dwf_ctx* c, int nconf, const double* theta)
{
    return set_gauge(c, nconf, theta, cudaMemcpyHostToDevice);
}

int dwf_set_gauge_dev(dwf_ctx* c, int nconf, const double* theta_dev)
{
    return set_gauge(c, nconf, theta_dev, cudaMemcpyDeviceToDevice);
}

int dwf_apply_dev(dwf_ctx* c, int op, int conf, const void* in, void* out, int nrhs, int precision)
{
    if (!c || !in || !out)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    return apply_dev(c, op, nrhs, nullptr, conf, in, out, precision);
}

int dwf_apply(dwf_ctx* c, int op, int conf, const double* in, double* out, int nrhs)
{
    if (!c || !in || !out || nrhs < 1)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    int st = ensure_workspace(c, nrhs);
    if (st)
        return st;
    const size_t bytes = size_t(nrhs) * c->fsz() * sizeof(double2);
    CK(cudaMemcpyAsync(c->w_b, in, bytes, cudaMemcpyHostToDevice, c->stream));
    st = apply_dev(c, op, nrhs, nullptr, conf, c->w_b, c->w_x, 64);
    if (st)
        return st;
    CK(cudaMemcpyAsync(out, c->w_x, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->dslash_err)
    {
        // a slice-ring Dslash wait that ran out (in this call or an earlier dwf_apply_dev)
        int e = 0;
        CK(cudaMemcpy(&e, c->dslash_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e != 0)
        {
            CK(cudaMemset(c->dslash_err, 0, sizeof(int)));
            return ctx_fail(c, e, "apply: a slice-ring Dslash copy wait ran out");
        }
    }
    return DWF_OK;
}

int dwf_cg_batch_dev(dwf_ctx* c, int op, int nrhs, const int* rhs_conf, const void* b, void* x,
                     int has_guess, double rtol, int maxiter, int solver, dwf_solve_info* info)
{
    if (!c || !b || !x)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    return solve_batch(c, op, nrhs, rhs_conf, static_cast<const double2*>(b),
                       static_cast<double2*>(x), has_guess, rtol, maxiter, solver,
                       c->kind == 1 ? 1 : 0, info);
}

int dwf_cg(dwf_ctx* c, int op, int conf, const double* b, double* x, int has_guess, double rtol,
           int maxiter, int solver, dwf_solve_info* info)
{
    if (!c || !b || !x)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    // The staging buffers w_b / w_x must not be reallocated by the solver:
    // size the workspace first.
    int st = ensure_workspace(c, 1);
    if (st)
        return st;
    const size_t bytes = c->fsz() * sizeof(double2);
    CK(cudaMemcpyAsync(c->w_b, b, bytes, cudaMemcpyHostToDevice, c->stream));
    if (has_guess)
        CK(cudaMemcpyAsync(c->w_x, x, bytes, cudaMemcpyHostToDevice, c->stream));
    st = solve_batch(c, op, 1, &conf, c->w_b, c->w_x, has_guess, rtol, maxiter, solver,
                     c->kind == 1 ? 1 : 0, info);
    if (st)
        return st;
    CK(cudaMemcpyAsync(x, c->w_x, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return info ? info->status : DWF_OK;
}

int dwf_cg_batch(dwf_ctx* c, int op, int nrhs, const int* rhs_conf, const double* b, double* x,
                 int has_guess, double rtol, int maxiter, int solver, dwf_solve_info* info)
{
    if (!c || !b || !x || nrhs < 1)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    int st = ensure_workspace(c, nrhs);
    if (st)
        return st;
    const size_t bytes = size_t(nrhs) * c->fsz() * sizeof(double2);
    CK(cudaMemcpyAsync(c->w_src, b, bytes, cudaMemcpyHostToDevice, c->stream));
    if (has_guess)
        CK(cudaMemcpyAsync(c->w_x, x, bytes, cudaMemcpyHostToDevice, c->stream));
    st = solve_batch(c, op, nrhs, rhs_conf, c->w_src, c->w_x, has_guess, rtol, maxiter, solver,
                     c->kind == 1 ? 1 : 0, info);
    if (st)
        return st;
    CK(cudaMemcpyAsync(x, c->w_x, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int dwf_propagators_dev(dwf_ctx* c, int nrhs, const int* rhs_conf, const void* src, void* x,
                        double rtol, int maxiter, int solver, dwf_solve_info* info)
{
    if (!c || !src || !x)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    return propagators(c, nrhs, rhs_conf, static_cast<const double2*>(src),
                       static_cast<double2*>(x), rtol, maxiter, solver, info);
}

int dwf_propagators(dwf_ctx* c, int nrhs, const int* rhs_conf, const double* src, double* x,
                    double rtol, int maxiter, int solver, dwf_solve_info* info)
{
    if (!c || !src || !x || nrhs < 1)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    int st = ensure_workspace(c, nrhs);
    if (st)
        return st;
    const size_t bytes = size_t(nrhs) * c->fsz() * sizeof(double2);
    // Even-odd cluster batches of at least two waves: solve in DWFB_PIPE_CHUNKS
    // chunks of whole waves, the sources of every chunk copied in and the
    // solutions of each finished chunk copied out on a second stream while
    // the next chunks solve (the copies overlap the solves when the host
    // buffers are page-locked). Each right-hand side's Schur solve is the one
    // a single batch would run; the full-lattice check is decided per chunk.
    const int wave = solver == DWF_SOLVER_EO_MIXED ? eo_cluster_wave(c) : 0;
    if (wave > 0 && nrhs >= 2 * wave)
        return propagators_pipelined(c, nrhs, rhs_conf, src, x, rtol, maxiter, solver, info,
                                     wave * ((nrhs + DWFB_PIPE_CHUNKS * wave - 1) / (DWFB_PIPE_CHUNKS * wave)));
    CK(cudaMemcpyAsync(c->w_src, src, bytes, cudaMemcpyHostToDevice, c->stream));
    st = propagators(c, nrhs, rhs_conf, c->w_src, c->w_x, rtol, maxiter, solver, info);
    if (st)
        return st;
    CK(cudaMemcpyAsync(x, c->w_x, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

uint64_t dwf_launch_count(const dwf_ctx* c) { return c ? c->launches : 0; }

int dwf_set_dslash_variant(dwf_ctx* c, int variant)
{
    if (!c || variant < -1 || variant > 6)
        return DWF_BAD_ARG;
    if (variant == 6 && !c->dslash_err)
    {
        // the slice-ring kernel's error word
        CK(cudaSetDevice(c->device));
        CK(cudaMalloc(&c->dslash_err, sizeof(int)));
        CK(cudaMemset(c->dslash_err, 0, sizeof(int)));
    }
    c->dslash_variant = variant;
    if (variant == -1)
        c->dslash_tuned.clear();
    return DWF_OK;
}

int dwf_set_dslash_chunk(dwf_ctx* c, int rows)
{
    if (!c || rows < 0)
        return DWF_BAD_ARG;
    c->dslash_chunk = rows;
    c->dslash_tuned.clear();
    return DWF_OK;
}

int dwf_dslash_variant(const dwf_ctx* c, int precision, int nrhs)
{
    if (!c || (precision != 64 && precision != 32) || nrhs < 1)
        return -1;
    if (c->dslash_variant >= 0)
        return c->dslash_variant;
    int bucket = 0;
    while ((1 << bucket) < nrhs && bucket < 20)
        ++bucket;
    const auto it = c->dslash_tuned.find((precision == 64 ? 100 : 0) + bucket);
    return it == c->dslash_tuned.end() ? -1 : it->second.variant;
}

int dwf_barrier_selftest(dwf_ctx* c, int missing_blocks, uint64_t limit_ns)
{
    if (!c || missing_blocks < 0 || limit_ns == 0)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    const unsigned grid = unsigned(std::max(1, c->nsm));
    CK(cudaMemsetAsync(c->bar, 0, sizeof(GridBar), c->stream));
    const unsigned expected = grid + unsigned(missing_blocks);
    unsigned long long lim = limit_ns;
    int rounds = 8;
    GridBar* bar = c->bar;
    void* args[] = {&bar, const_cast<unsigned*>(&expected), &lim, &rounds};
    CK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&barrier_probe_kernel), dim3(grid),
                                   dim3(32), args, 0, c->stream));
    c->launches += 1;
    GridBar hb{};
    CK(cudaMemcpyAsync(&hb, c->bar, sizeof(GridBar), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (hb.err != 0)
        return ctx_fail(c, hb.err, "grid barrier wait ran out");
    return DWF_OK;
}

double dwf_solver_kernel_ms(const dwf_ctx* c, int kind, uint64_t* nlaunch)
{
    if (!c || kind < 0 || kind > 2)
        return 0.0;
    if (nlaunch)
        *nlaunch = c->solver_launches[kind];
    return c->solver_ms[kind];
}

uint64_t dwf_graph_replays(const dwf_ctx* c, int* cached)
{
    if (!c)
        return 0;
    if (cached)
        *cached = int(c->graphs.size());
    return c->graph_replays;
}

}  // extern "C"
