// Learned preconditioner: PTC network kernels (forward / adjoint layers on
// the tensor cores, weight gradients, loss, Adam), GPU training on pairs that
// the plain solver generates, and the preconditioned solve.
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "learned.cuh"

using namespace dwfb;

#define CK(call)                                                                        \
    do                                                                                  \
    {                                                                                   \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ctx_fail(c, DWF_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

#define ST(call)                 \
    do                           \
    {                            \
        const int s_ = (call);   \
        if (s_ != DWF_OK)        \
            return s_;           \
    } while (0)

namespace dwfb {

// Offsets (dt, dx) of the 3x3 stencil.
__constant__ int kOffT[9] = {0, 1, -1, 0, 0, 1, 1, -1, -1};
__constant__ int kOffX[9] = {0, 0, 0, 1, -1, 1, -1, 1, -1};

// Field layout seen by a layer: complex element (rhs, site h, channel c) at
// rhs * rs + h * hs + (c / cg) * sg + (c % cg). Operator layout (domain wall
// ((s*Nt+t)*Nx+x)*2+spin, c = 2 s + spin): hs = 2, cg = 2, sg = 2V.
// Network layout [V][C]: hs = C, cg = C, sg = 0.
struct FieldLayout
{
    long rs;
    int hs, cg, sg;
};

__host__ __device__ __forceinline__ long chan_off(const FieldLayout& f, int c)
{
    return long(c / f.cg) * f.sg + (c % f.cg);
}

// ---------------------------------------------------------------------------
// transports
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 hop_t(const double2* U, const Lat& L, int t, int x, int sg)
{
    const int Nt = L.Nt, Nx = L.Nx;
    t = (t % Nt + Nt) % Nt;
    x = (x % Nx + Nx) % Nx;
    if (sg > 0)
    {
        const double2 u = U[t * Nx + x];
        const double s = (t == Nt - 1) ? L.bct : 1.0;
        return make_double2(s * u.x, s * u.y);
    }
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const double2 u = U[tm * Nx + x];
    const double s = (t == 0) ? L.bct : 1.0;
    return make_double2(s * u.x, -s * u.y);
}

__device__ __forceinline__ double2 hop_x(const double2* U, const Lat& L, int t, int x, int sg)
{
    const int Nt = L.Nt, Nx = L.Nx;
    t = (t % Nt + Nt) % Nt;
    x = (x % Nx + Nx) % Nx;
    const double2* Ux = U + L.V;
    if (sg > 0)
    {
        const double2 u = Ux[t * Nx + x];
        const double s = (x == Nx - 1) ? L.bcx : 1.0;
        return make_double2(s * u.x, s * u.y);
    }
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const double2 u = Ux[t * Nx + xm];
    const double s = (x == 0) ? L.bcx : 1.0;
    return make_double2(s * u.x, -s * u.y);
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// T[conf][h][k] (FP32) from the FP64 links of each configuration.
__global__ void lp_transport_kernel(Lat L, const double2* __restrict__ U64, long usz, int nconf,
                                    float2* __restrict__ T)
{
    const long n = long(nconf) * L.V;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const int cf = int(i / L.V);
        const int h = int(i - long(cf) * L.V);
        const int t = h / L.Nx, x = h - t * L.Nx;
        const double2* U = U64 + cf * usz;
        float2* out = T + i * 9;
        out[0] = make_float2(1.f, 0.f);
        for (int k = 1; k < 9; ++k)
        {
            const int dt = kOffT[k], dx = kOffX[k];
            double2 v;
            if (dx == 0)
                v = hop_t(U, L, t, x, dt);
            else if (dt == 0)
                v = hop_x(U, L, t, x, dx);
            else
            {
                const double2 p1 = zmul(hop_t(U, L, t, x, dt), hop_x(U, L, t + dt, x, dx));
                const double2 p2 = zmul(hop_x(U, L, t, x, dx), hop_t(U, L, t, x + dx, dt));
                v = make_double2(0.5 * (p1.x + p2.x), 0.5 * (p1.y + p2.y));
            }
            out[k] = make_float2(float(v.x), float(v.y));
        }
    }
}

// ---------------------------------------------------------------------------
// weight packing into mma.m16n8k16 B fragments
// ---------------------------------------------------------------------------
// The complex contraction P[o] = sum_j W[o][j] a[j] is the real product of
// A = [re a_j, im a_j]_j (interleaved) with B[2j][2o] = Re W, B[2j+1][2o] = -Im W,
// B[2j][2o+1] = Im W, B[2j+1][2o+1] = Re W. Input channels are padded to
// cpad (a multiple of 8) per offset; k-step ks covers offset k = ks / (cpad/8)
// and channels 8 (ks % (cpad/8)) .. +7. Fragment of lane (g = lane/4,
// q = lane%4) for k-step ks and n-tile nt: real column n = 8 nt + g (output
// o = n/2, part n%2), activation rows j = 8 ks + q (b0) and j + 4 (b1), the
// low half holding the row of Re a_j.
__device__ __forceinline__ uint32_t pack_bf2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__global__ void lp_pack_kernel(const float2* __restrict__ W, int cin, int cout, int adjoint,
                               int cpad, int nt, uint2* __restrict__ B)
{
    // layer dimensions as seen by the packed (possibly adjoint) layer
    const int ci = adjoint ? cout : cin;
    const int co = adjoint ? cin : cout;
    const int ksteps = 9 * cpad / 8;
    const int total = ksteps * nt * 32;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x)
    {
        const int lane = idx & 31;
        const int tile = idx >> 5;
        const int ks = tile / nt, ntile = tile - ks * nt;
        const int g = lane >> 2, q = lane & 3;
        const int n = 8 * ntile + g;
        const int o = n >> 1, part = n & 1;
        uint32_t r[2];
        for (int h = 0; h < 2; ++h)
        {
            const int j = 8 * ks + q + 4 * h;
            const int k = j / cpad, i = j - k * cpad;
            float2 w = make_float2(0.f, 0.f);
            if (o < co && i < ci)
            {
                if (!adjoint)
                    w = W[(long(k) * cout + o) * cin + i];
                else
                {
                    // W'_k[o][i] = conj(W_rev(k)[i][o])
                    const int kr = (k == 0) ? 0 : ((k <= 4) ? ((k & 1) ? k + 1 : k - 1) : 13 - k);
                    const float2 u = W[(long(kr) * cout + i) * cin + o];
                    w = make_float2(u.x, -u.y);
                }
            }
            r[h] = part == 0 ? pack_bf2(w.x, -w.y) : pack_bf2(w.y, w.x);
        }
        B[idx] = make_uint2(r[0], r[1]);
    }
}

// ---------------------------------------------------------------------------
// PTC layer as an implicit GEMM on the tensor cores
// ---------------------------------------------------------------------------
// out(y) = sum_k T_k(y) P_k(y + d_k), P_k = W_k in. A block owns a tile of
// kTileRows t-rows x tx x-sites of one right-hand side: it stages the input
// on the tile and its one-site halo in shared memory as BF16 (site-major,
// channels padded to cpad with a 4-word skew so ldmatrix rows hit distinct
// banks); each warp then computes 16 consecutive x-sites: per offset k the
// A fragments of the shifted window come from ldmatrix, the B fragments
// (weights) from shared memory, P_k accumulates in FP32 registers and is
// multiplied by the FP32 transporter of each row before it joins the sum.
struct ConvArgs
{
    const float2* in;
    float2* out;
    FieldLayout li, lo;
    int cin, cout, cpad;   // channels; input channels padded to a multiple of 8
    int tx;                // tile width in x (multiple of 16)
    const uint2* B;        // [9 * cpad / 8][NT][32]
    const float2* T;       // [nconf][V][9]
    const int* conf;
    int conf0;
    int Nt, Nx, V, nrhs;
};

constexpr int kConvWarps = 8;
constexpr int kTileRows = 2;

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const void* p)
{
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

__host__ __device__ __forceinline__ int conv_site_words(int cpad) { return cpad + 4; }

__host__ __device__ __forceinline__ size_t conv_smem_bytes(int cpad, int nt, int tx)
{
    return size_t(9) * (cpad / 8) * nt * 32 * sizeof(uint2) +
           size_t(kTileRows + 2) * (tx + 2) * conv_site_words(cpad) * sizeof(uint32_t);
}

template <int NT>
__global__ void __launch_bounds__(kConvWarps * 32) lp_conv_kernel(ConvArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* Bs = reinterpret_cast<uint2*>(smem);
    const int ks_per = a.cpad / 8;
    const int nb_frag = 9 * ks_per * NT * 32;
    uint32_t* tile = reinterpret_cast<uint32_t*>(Bs + nb_frag);
    const int SW = conv_site_words(a.cpad);
    const int TW = a.tx + 2;
    for (int i = threadIdx.x; i < nb_frag; i += blockDim.x)
        Bs[i] = a.B[i];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int rows_t = (a.Nt + kTileRows - 1) / kTileRows;
    const int cols_t = (a.Nx + a.tx - 1) / a.tx;
    const long ntiles = long(rows_t) * cols_t * a.nrhs;
    const int npairs = a.cpad / 2;  // channel pairs per site
    const int mt_per_row = a.tx / 16;
    for (long tl = blockIdx.x; tl < ntiles; tl += gridDim.x)
    {
        const int rhs = int(tl / (long(rows_t) * cols_t));
        const int rem = int(tl - long(rhs) * rows_t * cols_t);
        const int t0 = (rem / cols_t) * kTileRows;
        const int x0 = (rem - (rem / cols_t) * cols_t) * a.tx;
        const int cf = a.conf ? a.conf[rhs] : a.conf0;
        const float2* inr = a.in + long(rhs) * a.li.rs;
        __syncthreads();  // previous tile's readers are done
        // stage the input on the tile and its halo (2 channels per thread step)
        const int nstage = (kTileRows + 2) * TW * npairs;
        for (int e = threadIdx.x; e < nstage; e += blockDim.x)
        {
            const int site = e / npairs, cp = e - site * npairs;
            const int r = site / TW, cc = site - r * TW;
            int t = t0 - 1 + r, x = x0 - 1 + cc;
            t = t < 0 ? t + a.Nt : (t >= a.Nt ? t - a.Nt : t);
            x = x % a.Nx;  // x0 - 1 + cc >= -1
            x = x < 0 ? x + a.Nx : x;
            const int h = t * a.Nx + x;
            uint32_t w0 = 0u, w1 = 0u;
            const int c0 = 2 * cp;
            if (c0 < a.cin)
            {
                if (c0 + 1 < a.cin && chan_off(a.li, c0 + 1) == chan_off(a.li, c0) + 1)
                {
                    const float4 v = *reinterpret_cast<const float4*>(inr + long(h) * a.li.hs + chan_off(a.li, c0));
                    w0 = pack_bf2(v.x, v.y);
                    w1 = pack_bf2(v.z, v.w);
                }
                else
                {
                    const float2 v = inr[long(h) * a.li.hs + chan_off(a.li, c0)];
                    w0 = pack_bf2(v.x, v.y);
                    if (c0 + 1 < a.cin)
                    {
                        const float2 u = inr[long(h) * a.li.hs + chan_off(a.li, c0 + 1)];
                        w1 = pack_bf2(u.x, u.y);
                    }
                }
            }
            uint32_t* d = tile + site * SW + c0;
            d[0] = w0;
            d[1] = w1;
        }
        __syncthreads();
        const float2* Tc = a.T + long(cf) * a.V * 9;
        float2* outr = a.out + long(rhs) * a.lo.rs;
        for (int mt = warp; mt < kTileRows * mt_per_row; mt += kConvWarps)
        {
            const int r = mt / mt_per_row;
            const int xs = (mt - r * mt_per_row) * 16;
            const int t = t0 + r;
            const bool row_ok = t < a.Nt;
            const int xg0 = x0 + xs + g, xg1 = xg0 + 8;
            const bool ok0 = row_ok && xg0 < a.Nx, ok1 = row_ok && xg1 < a.Nx;
            const int h0 = t * a.Nx + xg0, h1 = t * a.Nx + xg1;
            float acc[NT][4];
#pragma unroll
            for (int n = 0; n < NT; ++n)
                acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
            for (int k = 0; k < 9; ++k)
            {
                const int dt = kOffT[k], dx = kOffX[k];
                // ldmatrix row of this lane: window site (r + 1 + dt, xs + 1 + dx + (lane & 15)),
                // channels 4 (lane / 16) .. +3 of each 8-channel k-step
                const uint32_t* wrow = tile + ((r + 1 + dt) * TW + xs + 1 + dx + (lane & 15)) * SW + (lane >> 4) * 4;
                float P[NT][4];
#pragma unroll
                for (int n = 0; n < NT; ++n)
                    P[n][0] = P[n][1] = P[n][2] = P[n][3] = 0.f;
                for (int ks = 0; ks < ks_per; ++ks)
                {
                    uint32_t A[4];
                    ldmatrix_x4(A, wrow + ks * 8);
                    const uint2* bp = Bs + ((k * ks_per + ks) * NT) * 32 + lane;
#pragma unroll
                    for (int n = 0; n < NT; ++n)
                    {
                        const uint2 b = bp[n * 32];
                        mma_bf16(P[n], A[0], A[1], A[2], A[3], b.x, b.y);
                    }
                }
                const float2 T0 = ok0 ? Tc[long(h0) * 9 + k] : make_float2(0.f, 0.f);
                const float2 T1 = ok1 ? Tc[long(h1) * 9 + k] : make_float2(0.f, 0.f);
#pragma unroll
                for (int n = 0; n < NT; ++n)
                {
                    acc[n][0] += T0.x * P[n][0] - T0.y * P[n][1];
                    acc[n][1] += T0.x * P[n][1] + T0.y * P[n][0];
                    acc[n][2] += T1.x * P[n][2] - T1.y * P[n][3];
                    acc[n][3] += T1.x * P[n][3] + T1.y * P[n][2];
                }
            }
#pragma unroll
            for (int n = 0; n < NT; ++n)
            {
                const int o = 4 * n + q;
                if (o < a.cout)
                {
                    const long off = chan_off(a.lo, o);
                    if (ok0)
                        outr[long(h0) * a.lo.hs + off] = make_float2(acc[n][0], acc[n][1]);
                    if (ok1)
                        outr[long(h1) * a.lo.hs + off] = make_float2(acc[n][2], acc[n][3]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// PTC layer on the 5th-generation tensor cores (tcgen05, accumulators in TMEM)
// ---------------------------------------------------------------------------
// Sites are addressed in padded rows: lattice row t holds P = Nx + 2 rows,
// row t P + 1 + x for site (t, x) and one halo row on each side (x = -1 and
// x = Nx, i.e. the wrapped neighbours). A CTA owns tiles of 128 consecutive
// padded rows of one right-hand side; the input around a tile (padded rows
// pr0 - P - 1 .. pr0 + 127 + P + 1) is staged once in shared memory as BF16,
// double-buffered across tiles, so that the operand of every offset
// (dt, dx) is the contiguous 128-row window starting (1 + dt) P + 1 + dx rows
// into the staged window (a row shift of the MMA's start address). Layout of
// the window: planes of 4 complex channels (16 B per row), the canonical
// no-swizzle K-major layout of tcgen05.mma (rows 16 B apart, 8-row groups
// 128 B apart, the two 16-B K-chunks of a k-step one plane apart). The
// weights are the B operand (N = 2 cout real columns, K-major). One elected
// thread issues, per offset, cpad/8 MMAs of 128 x N x 16 into one of four
// TMEM accumulators and commits them to an mbarrier; meanwhile the 4
// epilogue warps read a finished accumulator (tcgen05.ld, one row per
// thread), multiply by that row's FP32 transporter and add into FP32
// registers. Halo rows are computed and dropped.
struct TcArgs
{
    const float2* in;
    float2* out;
    FieldLayout li, lo;
    int cin, cout, cpad, ncol;   // ncol: real output columns (multiple of 16)
    const uint4* B;              // [9 cpad/8][2][ncol] x 8 BF16
    const float2* T;
    const int* conf;
    int conf0;
    int Nt, Nx, V, nrhs;
    int* err;
    unsigned long long timeout_ns;
    // BF16 planar fields ([rhs][plane][site] x 16 B, 4 channels per plane):
    // when set, the input is read from in_bf (cp.async) instead of `in`, and
    // the output written to out_bf instead of `out`
    const uint4* in_bf;
    uint4* out_bf;
    int nbuf;   // window buffers per CTA (1: two CTAs share an SM; 2: one CTA, double-buffered)
};

constexpr int kTcM = 128;

#ifndef DWFB_TC_PDL
#define DWFB_TC_PDL 1  // layer kernels launched as programmatic dependents of their predecessor
#endif

// Staged window of one tile in padded rows: lattice rows stored with one
// halo site on each side (P = Nx + 2 rows per lattice row), the tile's 128
// rows plus one padded lattice row and one site on each side.
__host__ __device__ __forceinline__ int tc_window_rows(int Nx) { return kTcM + 2 * (Nx + 2) + 2; }

__host__ __device__ __forceinline__ size_t tc_smem_bytes(int cpad, int ncol, int Nx, int nbuf)
{
    return size_t(9) * (cpad / 8) * 2 * ncol * 16 + size_t(nbuf) * (cpad / 4) * tc_window_rows(Nx) * 16;
}

// TMEM columns one CTA allocates (kSlots accumulators of ncol columns, a power of 2 >= 64).
__host__ __device__ constexpr uint32_t tc_tmem_cols(int ncol)
{
    return (4 * ncol <= 64) ? 64u : (4 * ncol <= 128) ? 128u : (4 * ncol <= 256) ? 256u : 512u;
}

// Tiles of 128 padded rows per right-hand side.
__host__ __device__ __forceinline__ long tc_tiles_per_rhs(int Nt, int Nx)
{
    return (long(Nt) * (Nx + 2) + kTcM - 1) / kTcM;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle (start, leading and stride byte
// offsets in 16-B units; version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u),
          "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, unsigned long long limit_ns)
{
    const unsigned long long t0 = globaltimer_ns();
    while (true)
    {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done)
            return true;
        if (globaltimer_ns() - t0 > limit_ns)
            return false;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

#define DWFB_R8(i) "=r"(v[i]), "=r"(v[i + 1]), "=r"(v[i + 2]), "=r"(v[i + 3]), "=r"(v[i + 4]), \
                   "=r"(v[i + 5]), "=r"(v[i + 6]), "=r"(v[i + 7])

// 32 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
        "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : DWFB_R8(0), DWFB_R8(8), DWFB_R8(16), DWFB_R8(24)
        : "r"(taddr));
}
#undef DWFB_R8

#define DWFB_R8(i) "=r"(v[i]), "=r"(v[i + 1]), "=r"(v[i + 2]), "=r"(v[i + 3]), "=r"(v[i + 4]), \
                   "=r"(v[i + 5]), "=r"(v[i + 6]), "=r"(v[i + 7])
// 16 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
        "%15}, [%16];\n"
        : DWFB_R8(0), DWFB_R8(8)
        : "r"(taddr));
}
#undef DWFB_R8

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

constexpr int kTcThreads = 256;

// Load 4 consecutive channels (one 16-B plane entry, BF16) of site h.
__device__ __forceinline__ uint4 load_plane(const float2* __restrict__ inr, const FieldLayout& L, int cin,
                                            long h, int c0)
{
    uint32_t w[4];
    if (c0 + 3 < cin && L.cg % 4 == 0)
    {
        // 4 channels contiguous (network layout)
        const float4* p = reinterpret_cast<const float4*>(inr + h * L.hs + chan_off(L, c0));
        const float4 u = p[0], v = p[1];
        w[0] = pack_bf2(u.x, u.y);
        w[1] = pack_bf2(u.z, u.w);
        w[2] = pack_bf2(v.x, v.y);
        w[3] = pack_bf2(v.z, v.w);
    }
    else
    {
#pragma unroll
        for (int q = 0; q < 4; q += 2)
        {
            const int c = c0 + q;
            w[q] = w[q + 1] = 0u;
            if (c + 1 < cin && L.cg % 2 == 0)
            {
                // channel pair contiguous (operator layout: the two spins of one slice)
                const float4 u = *reinterpret_cast<const float4*>(inr + h * L.hs + chan_off(L, c));
                w[q] = pack_bf2(u.x, u.y);
                w[q + 1] = pack_bf2(u.z, u.w);
            }
            else if (c < cin)
            {
                const float2 u = inr[h * L.hs + chan_off(L, c)];
                w[q] = pack_bf2(u.x, u.y);
                if (c + 1 < cin)
                {
                    const float2 u1 = inr[h * L.hs + chan_off(L, c + 1)];
                    w[q + 1] = pack_bf2(u1.x, u1.y);
                }
            }
        }
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// Wait for the phase of `parity` of an mbarrier: poll (try_wait suspends
// between polls), reading the timer only every 64 polls; false on timeout.
__device__ __forceinline__ bool mbar_wait_lean(uint32_t mbar, uint32_t parity, unsigned long long limit_ns)
{
    unsigned long long t0 = 0;
    for (int it = 0;; ++it)
    {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done)
            return true;
        if ((it & 63) == 0)
        {
            const unsigned long long t = globaltimer_ns();
            if (it == 0)
                t0 = t;
            else if (t - t0 > limit_ns)
                return false;
        }
    }
}

// Warp roles of the tcgen05 layer kernel (kTcThreads = 256):
//   warps 0-3  epilogue: one TMEM lane (output row) per thread, all columns
//   warp 4     MMA issue (one elected thread)
//   warps 5-7  producers: stage the window of tile n into buffer n % nbuf as
//              soon as the MMAs of tile n - nbuf are done with it
// mbarriers: tfull[s] / tempty[s] per TMEM slot, wfull[b] / wfree[b] per
// window buffer.
constexpr int kEpiWarps = 4;
constexpr int kProdWarps = 3;

template <int NCOL>
__global__ void __launch_bounds__(kTcThreads, 2) lp_tc_kernel(TcArgs a)
{
    extern __shared__ __align__(128) unsigned char tc_smem[];
    constexpr int kSlots = 4;
    __shared__ __align__(8) uint64_t mbar[2 * kSlots + 6];
    __shared__ uint32_t tmem_holder;
    constexpr int NC = NCOL / 2;
    static_assert(kSlots == 4, "tc_tmem_cols assumes four accumulator slots");
    constexpr uint32_t kCols = tc_tmem_cols(NCOL);
    static_assert(NC >= 1 && kSlots * NCOL <= 512, "TMEM columns");
    const int ksp = a.cpad / 8;
    const int nks = 9 * ksp;
    const int planes = a.cpad / 4;
    const int P = a.Nx + 2;                 // padded rows per lattice row
    const int J = tc_window_rows(a.Nx);     // staged rows per tile
    const long NP = long(a.Nt) * P;         // padded rows per right-hand side
    uint4* Bs = reinterpret_cast<uint4*>(tc_smem);
    uint4* As = Bs + nks * 2 * NCOL;        // [buffer][plane][row]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t mb = smem_u32(&mbar[0]);
    auto TFULL = [&](int sl) { return mb + 8u * uint32_t(sl); };
    auto TEMPTY = [&](int sl) { return mb + 8u * uint32_t(kSlots + sl); };
    auto WFULL = [&](int b) { return mb + 8u * uint32_t(2 * kSlots + b); };
    auto WFREE = [&](int b) { return mb + 8u * uint32_t(2 * kSlots + 2 + b); };
    for (int i = tid; i < nks * 2 * NCOL; i += blockDim.x)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(Bs + i)), "l"(a.B + i) : "memory");
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (tid == 0)
    {
        for (int i = 0; i < kSlots; ++i)
        {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(TFULL(i)), "r"(1u));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(TEMPTY(i)), "r"(uint32_t(kEpiWarps)));
        }
        for (int b = 0; b < 2; ++b)
        {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(WFULL(b)), "r"(uint32_t(kProdWarps * 32)));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(WFREE(b)), "r"(1u));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_holder)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_holder;
    // Launched as a programmatic dependent of the previous kernel on the
    // stream, the prologue above (weights, barriers, TMEM) may run while that
    // kernel finishes; every thread waits here for its completion before any
    // field is read or written, then lets the next layer's CTAs start their own
    // prologue (they take an SM only as this grid's CTAs leave it).
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const long tiles_per_rhs = tc_tiles_per_rhs(a.Nt, a.Nx);
    const long ntiles = tiles_per_rhs * a.nrhs;
    bool ok = true;

    if (warp >= kEpiWarps + 1)
    {
        // ---- producers ----
        const int pt = tid - (kEpiWarps + 1) * 32;  // 0 .. 95
        const int nprod = kProdWarps * 32;
        uint32_t free_ph = 0u;  // bit b: next wfree phase
        long it = 0;
        for (long tl = blockIdx.x; tl < ntiles; tl += gridDim.x, ++it)
        {
            const int rhs = int(tl / tiles_per_rhs);
            const long pr0 = (tl - long(rhs) * tiles_per_rhs) * kTcM;
            const int bf = int(it % a.nbuf);
            if (it >= a.nbuf)
            {
                // the MMAs of tile it - nbuf are done with this buffer
                if (!mbar_wait_lean(WFREE(bf), (free_ph >> bf) & 1u, a.timeout_ns))
                    ok = false;
                free_ph ^= 1u << bf;
            }
            uint4* Ab = As + long(bf) * planes * J;
            for (int j = pt; j < J; j += nprod)
            {
                // padded row pr0 - P - 1 + j, wrapped over the lattice's rows
                long pr = (pr0 - P - 1 + j) % NP;
                pr = pr < 0 ? pr + NP : pr;
                const int t = int(pr / P), xp = int(pr - long(t) * P);
                const int x = (xp == 0) ? a.Nx - 1 : ((xp == P - 1) ? 0 : xp - 1);
                const int src = t * a.Nx + x;
                if (a.in_bf)
                {
                    const uint4* base = a.in_bf + long(rhs) * planes * a.V + src;
                    for (int pl = 0; pl < planes; ++pl)
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                         smem_u32(Ab + pl * J + j)),
                                     "l"(base + long(pl) * a.V)
                                     : "memory");
                }
                else
                {
                    const float2* inr = a.in + long(rhs) * a.li.rs;
                    for (int pl = 0; pl < planes; ++pl)
                        Ab[pl * J + j] = load_plane(inr, a.li, a.cin, src, 4 * pl);
                }
            }
            if (a.in_bf)
            {
                // arrives once this thread's copies have landed
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(WFULL(bf)) : "memory");
            }
            else
            {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive(WFULL(bf));
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    else if (warp == kEpiWarps)
    {
        // ---- MMA issue ----
        if (lane == 0)
        {
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(NCOL >> 3) << 17) |
                                   (uint32_t(kTcM >> 4) << 24);
            const uint32_t a_base = smem_u32(As), b_base = smem_u32(Bs);
            const uint32_t a_lbo = uint32_t(J) * 16u;
            const uint32_t b_lbo = uint32_t(NCOL) * 16u;
            uint32_t full_ph = 0u;   // bit b: next wfull phase
            uint32_t empty_ph = 0u;  // bit s: next tempty phase
            uint32_t used = 0u;
            uint32_t g = 0;          // offsets issued so far
            long it = 0;
            for (long tl = blockIdx.x; tl < ntiles; tl += gridDim.x, ++it)
            {
                const int bf = int(it % a.nbuf);
                if (!mbar_wait_lean(WFULL(bf), (full_ph >> bf) & 1u, a.timeout_ns))
                    ok = false;
                full_ph ^= 1u << bf;
                // the producers' copies become visible to the tensor cores
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const uint32_t wbase = a_base + uint32_t(bf * planes * J) * 16u;
                for (int k = 0; k < 9; ++k, ++g)
                {
                    const int sl = int(g % kSlots);
                    if (used & (1u << sl))
                    {
                        if (!mbar_wait_lean(TEMPTY(sl), (empty_ph >> sl) & 1u, a.timeout_ns))
                            ok = false;
                        empty_ph ^= 1u << sl;
                    }
                    used |= 1u << sl;
                    tc_fence_after();
                    // window row of output row 0 for this offset
                    const int row0 = (1 + kOffT[k]) * P + 1 + kOffX[k];
                    const uint32_t d_tmem = tmem + uint32_t(sl) * uint32_t(NCOL);
                    for (int ks = 0; ks < ksp; ++ks)
                    {
                        const uint32_t aaddr = wbase + uint32_t((2 * ks) * J + row0) * 16u;
                        const uint32_t baddr = b_base + uint32_t((k * ksp + ks) * 2 * NCOL) * 16u;
                        tc_mma(d_tmem, umma_desc(aaddr, a_lbo, 128u), umma_desc(baddr, b_lbo, 128u), idesc,
                               ks > 0 ? 1u : 0u);
                    }
                    tc_commit(TFULL(sl));
                }
                tc_commit(WFREE(bf));
            }
            // the buffer-release arrivals of the last tiles land before the CTA exits
            const long mine = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
            for (int bf = 0; bf < a.nbuf; ++bf)
            {
                const long uses = (mine + a.nbuf - 1 - bf) / a.nbuf;   // tiles that used buffer bf
                if (uses > 0 && !mbar_wait_lean(WFREE(bf), uint32_t((uses - 1) & 1), a.timeout_ns))
                    ok = false;
            }
        }
        __syncwarp();
    }
    else
    {
        // ---- epilogue ----
        const int erow = 32 * warp + lane;
        uint32_t full_ph = 0u;  // bit s: next tfull phase
        uint32_t g = 0;
        for (long tl = blockIdx.x; tl < ntiles; tl += gridDim.x)
        {
            const int rhs = int(tl / tiles_per_rhs);
            const long pr = (tl - long(rhs) * tiles_per_rhs) * kTcM + erow;   // this thread's padded row
            const int cf = a.conf ? a.conf[rhs] : a.conf0;
            const int tr = int(pr / P), xp = int(pr - long(tr) * P);
            // halo rows (xp = 0, P - 1) and rows past the lattice are dropped
            const bool row_ok = pr < NP && xp >= 1 && xp <= a.Nx;
            const int hrow = row_ok ? tr * a.Nx + xp - 1 : 0;
            float2 Tk[9];
            {
                const float2* Tc = a.T + (long(cf) * a.V + (row_ok ? hrow : 0)) * 9;
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    Tk[q] = row_ok ? Tc[q] : make_float2(0.f, 0.f);
            }
            float acc[NC][2];
#pragma unroll
            for (int cc = 0; cc < NC; ++cc)
                acc[cc][0] = acc[cc][1] = 0.f;
#pragma unroll 1
            for (int q = 0; q < 9; ++q, ++g)
            {
                const int sl = int(g % kSlots);
                if (!mbar_wait_lean(TFULL(sl), (full_ph >> sl) & 1u, a.timeout_ns))
                    ok = false;
                full_ph ^= 1u << sl;
                tc_fence_after();
                const int k = q;   // the MMAs run the offsets in order
                float2 T = Tk[0];
#pragma unroll
                for (int u = 1; u < 9; ++u)
                    T = (k == u) ? Tk[u] : T;
                const uint32_t tbase = tmem + (uint32_t(32 * warp) << 16) + uint32_t(sl * NCOL);
#pragma unroll
                for (int c0 = 0; c0 < NCOL; c0 += 32)
                {
                    uint32_t v[32];
                    if (c0 + 32 <= NCOL)
                        tmem_ld32(tbase + uint32_t(c0), v);
                    else
                    {
                        uint32_t w[16];
                        tmem_ld16(tbase + uint32_t(c0), w);
#pragma unroll
                        for (int u = 0; u < 16; ++u)
                            v[u] = w[u];
                    }
                    tmem_wait_ld();
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                    {
                        if (c0 / 2 + u < NC)
                        {
                            const float pr = __uint_as_float(v[2 * u]), pi = __uint_as_float(v[2 * u + 1]);
                            acc[c0 / 2 + u][0] += T.x * pr - T.y * pi;
                            acc[c0 / 2 + u][1] += T.x * pi + T.y * pr;
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0)
                    mbar_arrive(TEMPTY(sl));
            }
            if (row_ok)
            {
                if (a.out_bf)
                {
                    const int planes_out = (a.cout + 7) / 8 * 2;
                    uint4* ob = a.out_bf + long(rhs) * planes_out * a.V + hrow;
#pragma unroll
                    for (int cc = 0; cc < NC; cc += 4)
                    {
                        uint32_t w[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            w[u] = (cc + u < a.cout && cc + u < NC) ? pack_bf2(acc[cc + u][0], acc[cc + u][1]) : 0u;
                        if (cc / 4 < planes_out)
                            ob[long(cc / 4) * a.V] = make_uint4(w[0], w[1], w[2], w[3]);
                    }
                }
                else
                {
                    float2* outr = a.out + long(rhs) * a.lo.rs + long(hrow) * a.lo.hs;
#pragma unroll
                    for (int cc = 0; cc < NC; ++cc)
                        if (cc < a.cout)
                            outr[chan_off(a.lo, cc)] = make_float2(acc[cc][0], acc[cc][1]);
                }
            }
        }
    }
    if (!ok && a.err)
        atomicExch(a.err, DWF_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// FP32 field (any layout) -> BF16 planar [rhs][plane][site].
__global__ void lp_to_planar_kernel(const float2* __restrict__ in, FieldLayout L, int cin, int planes, int V,
                                    int nrhs, uint4* __restrict__ out)
{
    const long n = long(nrhs) * planes * V;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const int h = int(i % V);
        const long r = i / V;
        const int pl = int(r % planes), rhs = int(r / planes);
        out[i] = load_plane(in + long(rhs) * L.rs, L, cin, h, 4 * pl);
    }
}

// Weights in the tcgen05 B layout: element (k-step ks, K-chunk ch, column n,
// e) is BF16 number 8 ch + e of the k-step's reduction index (activation
// j = 8 ks + (8 ch + e) / 2, real part for even e) against real column n.
__global__ void lp_pack_tc_kernel(const float2* __restrict__ W, int cin, int cout, int adjoint, int cpad,
                                  int ncol, __nv_bfloat16* __restrict__ B)
{
    const int ci = adjoint ? cout : cin;
    const int co = adjoint ? cin : cout;
    const int nks = 9 * cpad / 8;
    const long total = long(nks) * 2 * ncol * 8;
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < total; idx += long(gridDim.x) * blockDim.x)
    {
        const int e = int(idx & 7);
        const long r = idx >> 3;
        const int n = int(r % ncol);
        const int ch = int((r / ncol) & 1);
        const int ks = int(r / (2L * ncol));
        const int kk = 8 * ch + e;
        const int j = 8 * ks + (kk >> 1);
        const int k = j / cpad, i = j - k * cpad;
        const int o = n >> 1;
        float2 w = make_float2(0.f, 0.f);
        if (o < co && i < ci)
        {
            if (!adjoint)
                w = W[(long(k) * cout + o) * cin + i];
            else
            {
                const int kr = (k == 0) ? 0 : ((k <= 4) ? ((k & 1) ? k + 1 : k - 1) : 13 - k);
                const float2 u = W[(long(kr) * cout + i) * cin + o];
                w = make_float2(u.x, -u.y);
            }
        }
        float val;
        if ((n & 1) == 0)
            val = (kk & 1) ? -w.y : w.x;
        else
            val = (kk & 1) ? w.x : w.y;
        B[idx] = __float2bfloat16_rn(val);
    }
}

// ---------------------------------------------------------------------------
// weight gradient: G_k[o][i] = sum_{rhs, y} g(y)[o] conj(a_k(y)[i])
// ---------------------------------------------------------------------------
struct GradArgs
{
    const float2* in;   // layer input
    const float2* g;    // gradient at the layer output
    FieldLayout li, lg;
    int cin, cout;
    const float2* T;
    const int* conf;
    int conf0;
    int Nt, Nx, V, nrhs;
    float2* part;  // [gridDim.x][9][cout][cin]
};

constexpr int kGradSites = 32;
constexpr int kGradThreads = 256;
// weights per thread: cout * cin <= kGradThreads * PER; 4 for layers up to
// 1024 complex weights per offset, 6 up to 1536 (48 x 32: Ls = 24, 32 hidden)
constexpr int kGradMaxPer = 6;

template <int PER>
__global__ void __launch_bounds__(kGradThreads) lp_wgrad_kernel(GradArgs a)
{
    constexpr int kGradMaxPer = PER;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* gs = reinterpret_cast<float2*>(smem);      // [32][cout]
    float2* as = gs + kGradSites * a.cout;             // [32][cin]
    const int E = a.cout * a.cin;
    float2 acc[9][kGradMaxPer];
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
        for (int m = 0; m < kGradMaxPer; ++m)
            acc[k][m] = make_float2(0.f, 0.f);
    const int chunks_per_rhs = (a.V + kGradSites - 1) / kGradSites;
    const long nchunks = long(chunks_per_rhs) * a.nrhs;
    for (long chn = blockIdx.x; chn < nchunks; chn += gridDim.x)
    {
        const int rhs = int(chn / chunks_per_rhs);
        const int h0 = int(chn - long(rhs) * chunks_per_rhs) * kGradSites;
        const int cf = a.conf ? a.conf[rhs] : a.conf0;
        const float2* Tc = a.T + long(cf) * a.V * 9;
        const float2* inr = a.in + long(rhs) * a.li.rs;
        const float2* gr = a.g + long(rhs) * a.lg.rs;
        __syncthreads();
        for (int e = threadIdx.x; e < kGradSites * a.cout; e += blockDim.x)
        {
            const int r = e / a.cout, o = e - r * a.cout;
            const int h = h0 + r;
            gs[e] = (h < a.V) ? gr[long(h) * a.lg.hs + chan_off(a.lg, o)] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k)
        {
            __syncthreads();
            for (int e = threadIdx.x; e < kGradSites * a.cin; e += blockDim.x)
            {
                const int r = e / a.cin, i = e - r * a.cin;
                const int h = h0 + r;
                float2 v = make_float2(0.f, 0.f);
                if (h < a.V)
                {
                    const int t = h / a.Nx, x = h - t * a.Nx;
                    int tt = t + kOffT[k], xx = x + kOffX[k];
                    tt = tt < 0 ? tt + a.Nt : (tt >= a.Nt ? tt - a.Nt : tt);
                    xx = xx < 0 ? xx + a.Nx : (xx >= a.Nx ? xx - a.Nx : xx);
                    const float2 T = Tc[long(h) * 9 + k];
                    const float2 u = inr[long(tt * a.Nx + xx) * a.li.hs + chan_off(a.li, i)];
                    const uint32_t b = pack_bf2(u.x, u.y);
                    const float2 ub = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&b));
                    v = make_float2(T.x * ub.x - T.y * ub.y, T.x * ub.y + T.y * ub.x);
                }
                as[e] = v;
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < kGradMaxPer; ++m)
            {
                const int e = threadIdx.x + m * kGradThreads;
                if (e < E)
                {
                    const int o = e / a.cin, i = e - o * a.cin;
                    float2 s = acc[k][m];
                    for (int r = 0; r < kGradSites; ++r)
                    {
                        const float2 gv = gs[r * a.cout + o];
                        const float2 av = as[r * a.cin + i];
                        // g * conj(a)
                        s.x += gv.x * av.x + gv.y * av.y;
                        s.y += gv.y * av.x - gv.x * av.y;
                    }
                    acc[k][m] = s;
                }
            }
        }
    }
    float2* p = a.part + long(blockIdx.x) * 9 * E;
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
        for (int m = 0; m < kGradMaxPer; ++m)
        {
            const int e = threadIdx.x + m * kGradThreads;
            if (e < E)
                p[k * E + e] = acc[k][m];
        }
}

// grad[e] = sum over blocks of part[b][e], in FP64 and block order.
__global__ void lp_grad_reduce_kernel(const float2* __restrict__ part, int nblk, int n,
                                      float2* __restrict__ grad)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    {
        double sx = 0.0, sy = 0.0;
        for (int b = 0; b < nblk; ++b)
        {
            const float2 v = part[long(b) * n + e];
            sx += v.x;
            sy += v.y;
        }
        grad[e] = make_float2(float(sx), float(sy));
    }
}

// ---------------------------------------------------------------------------
// loss: (1/B) sum_b |out_b - e_b|^2 / |e_b|^2 and g = 2 (out - e) / (B |e_b|^2)
// ---------------------------------------------------------------------------
__global__ void lp_loss_partials_kernel(const float2* __restrict__ out, const float2* __restrict__ e,
                                        long fsz, int nblk, double* __restrict__ part)
{
    __shared__ double red[32];
    const int rhs = blockIdx.y;
    const long ch = (fsz + nblk - 1) / nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < fsz) ? i0 + ch : fsz;
    double dd = 0.0, ee = 0.0;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    {
        const float2 o = out[rhs * fsz + i], t = e[rhs * fsz + i];
        const double dx = double(o.x) - t.x, dy = double(o.y) - t.y;
        dd += dx * dx + dy * dy;
        ee += double(t.x) * t.x + double(t.y) * t.y;
    }
    dd = block_sum(dd, red);
    ee = block_sum(ee, red);
    if (threadIdx.x == 0)
    {
        part[(long(rhs) * nblk + blockIdx.x) * 2] = dd;
        part[(long(rhs) * nblk + blockIdx.x) * 2 + 1] = ee;
    }
}

// One thread per right-hand side: scale[b] = 2 / (B |e_b|^2), and (thread 0
// after a block-wide pass) the loss.
__global__ void lp_loss_finish_kernel(const double* __restrict__ part, int nrhs, int nblk,
                                      double* __restrict__ scale, double* __restrict__ loss)
{
    __shared__ double terms[1024];
    for (int b = threadIdx.x; b < nrhs; b += blockDim.x)
    {
        double dd = 0.0, ee = 0.0;
        for (int j = 0; j < nblk; ++j)
        {
            dd += part[(long(b) * nblk + j) * 2];
            ee += part[(long(b) * nblk + j) * 2 + 1];
        }
        scale[b] = 2.0 / (double(nrhs) * ee);
        if (b < 1024)
            terms[b] = dd / ee;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double s = 0.0;
        for (int b = 0; b < nrhs && b < 1024; ++b)
            s += terms[b];
        *loss = s / nrhs;
    }
}

__global__ void lp_loss_grad_kernel(const float2* __restrict__ out, const float2* __restrict__ e,
                                    long fsz, int nrhs, const double* __restrict__ scale,
                                    float2* __restrict__ g)
{
    const long n = fsz * nrhs;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const float s = float(scale[i / fsz]);
        const float2 o = out[i], t = e[i];
        g[i] = make_float2(s * (o.x - t.x), s * (o.y - t.y));
    }
}

// ---------------------------------------------------------------------------
// Adam on the FP32 master weights (real and imaginary parts separately)
// ---------------------------------------------------------------------------
__global__ void lp_adam_kernel(float* __restrict__ w, const float* __restrict__ g,
                               float* __restrict__ m, float* __restrict__ v, long n, float lr,
                               float b1, float b2, float c1, float c2, float eps)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// ---------------------------------------------------------------------------
// Gaussian fields from a counter-based generator (splitmix64 finaliser,
// Box-Muller): each complex component N(0, 1/2), as the pseudofermion draws.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void lp_gauss_kernel(double2* __restrict__ out, long n, uint64_t seed)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const uint64_t r = mix64(seed ^ mix64(uint64_t(i)));
        const double u1 = (double((r >> 11) & ((1ull << 26) - 1)) + 0.5) / double(1ull << 26);
        const double u2 = double(r >> 37) / double(1ull << 27);
        const double rad = sqrt(-log(u1));  // |z|^2 exponential with mean 1
        double s, co;
        sincospi(2.0 * u2, &s, &co);
        out[i] = make_double2(rad * co, rad * s);
    }
}

// ---------------------------------------------------------------------------
// vector kernels of the solver (FP32 fields, FP64 dot products)
// ---------------------------------------------------------------------------
struct Dot
{
    const float2* a;
    const float2* b;
};

// part[((slot * nrhs + rhs) * nblk + blk)] = <a, b> over this block's chunk,
// for up to three pairs, in one pass over the data.
__global__ void lp_dots_kernel(Dot d0, Dot d1, Dot d2, int ndot, long fsz, int nblk,
                               double2* __restrict__ part)
{
    __shared__ double red[32];
    const int rhs = blockIdx.y;
    const int nrhs = gridDim.y;
    const long ch = (fsz + nblk - 1) / nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < fsz) ? i0 + ch : fsz;
    const long base = long(rhs) * fsz;
    double re[3] = {0.0, 0.0, 0.0}, im[3] = {0.0, 0.0, 0.0};
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    {
#pragma unroll
        for (int s = 0; s < 3; ++s)
        {
            if (s < ndot)
            {
                const Dot d = s == 0 ? d0 : (s == 1 ? d1 : d2);
                const float2 x = d.a[base + i], y = d.b[base + i];
                re[s] += double(x.x) * y.x + double(x.y) * y.y;
                im[s] += double(x.x) * y.y - double(x.y) * y.x;
            }
        }
    }
    for (int s = 0; s < ndot; ++s)
    {
        const double r = block_sum(re[s], red);
        const double m = block_sum(im[s], red);
        if (threadIdx.x == 0)
            part[(long(s) * nrhs + rhs) * nblk + blockIdx.x] = make_double2(r, m);
    }
}

__device__ __forceinline__ double2 sum_part(const double2* part, int slot, int nrhs, int rhs, int nblk)
{
    double re = 0.0, im = 0.0;
    const double2* p = part + (long(slot) * nrhs + rhs) * nblk;
    for (int b = 0; b < nblk; ++b)
    {
        re += p[b].x;
        im += p[b].y;
    }
    return make_double2(re, im);
}

__device__ __forceinline__ double2 zdiv(double2 a, double2 b)
{
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

__device__ __forceinline__ bool zfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// Per-right-hand-side BiCGStab state.
struct BsState
{
    double2 rho, alpha, omega, beta;
    double rr;        // |r|^2 of the inner (normalised) system
    int active;       // 1 while iterating
    int breakdown;    // 1 once a denominator vanished
    int iters;
};

// Coefficient steps: 0 start (rho = <rh, r> from slot 0, rr from slot 1),
// 1 beta (rho1 = <rh, r>, rr = |r|^2 from slots 0, 1), 2 alpha (<rh, v> slot 0),
// 3 omega (<t, s> slot 0, <t, t> slot 1). tgt2: |r|^2 at which a right-hand
// side stops; maxit: inner iteration limit.
__global__ void lp_bs_coef_kernel(int step, const double2* __restrict__ part, int nrhs, int nblk,
                                  BsState* __restrict__ S, double tgt2, int maxit)
{
    const int rhs = blockIdx.x * blockDim.x + threadIdx.x;
    if (rhs >= nrhs)
        return;
    BsState st = S[rhs];
    if (step == 0)
    {
        st.rho = sum_part(part, 0, nrhs, rhs, nblk);
        st.rr = sum_part(part, 1, nrhs, rhs, nblk).x;
        st.alpha = make_double2(1.0, 0.0);
        st.omega = make_double2(1.0, 0.0);
        st.beta = make_double2(0.0, 0.0);
        st.breakdown = 0;
        st.iters = 0;
        st.active = st.active && st.rr > tgt2;
        S[rhs] = st;
        return;
    }
    if (!st.active)
    {
        st.alpha = st.omega = st.beta = make_double2(0.0, 0.0);
        S[rhs] = st;
        return;
    }
    if (step == 1)
    {
        const double2 rho1 = sum_part(part, 0, nrhs, rhs, nblk);
        st.rr = sum_part(part, 1, nrhs, rhs, nblk).x;
        if (st.rr <= tgt2 || st.iters >= maxit)
        {
            st.active = 0;
            st.alpha = st.omega = st.beta = make_double2(0.0, 0.0);
            S[rhs] = st;
            return;
        }
        // beta = (rho1 / rho) (alpha / omega)
        const double2 b = zmul(zdiv(rho1, st.rho), zdiv(st.alpha, st.omega));
        if (!zfinite(b) || (rho1.x == 0.0 && rho1.y == 0.0))
        {
            st.breakdown = 1;
            st.active = 0;
            st.alpha = st.omega = st.beta = make_double2(0.0, 0.0);
        }
        else
        {
            st.beta = b;
            st.rho = rho1;
        }
        st.iters += 1;
    }
    else if (step == 2)
    {
        const double2 a = zdiv(st.rho, sum_part(part, 0, nrhs, rhs, nblk));
        if (!zfinite(a))
        {
            st.breakdown = 1;
            st.active = 0;
            st.alpha = st.omega = st.beta = make_double2(0.0, 0.0);
        }
        else
            st.alpha = a;
    }
    else
    {
        const double2 ts = sum_part(part, 0, nrhs, rhs, nblk);
        const double tt = sum_part(part, 1, nrhs, rhs, nblk).x;
        double2 w = make_double2(ts.x / tt, ts.y / tt);
        if (!zfinite(w) || (w.x == 0.0 && w.y == 0.0))
        {
            // keep the alpha step (x += alpha ph, r = s), then stop
            st.breakdown = 1;
            w = make_double2(0.0, 0.0);
        }
        st.omega = w;
    }
    S[rhs] = st;
}

__device__ __forceinline__ float2 fz(double2 a) { return make_float2(float(a.x), float(a.y)); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// op 0: p = r + beta (p - omega v)
// op 1: s = r - alpha v
// op 2: x += alpha ph + omega sh ; r = s - omega t
__global__ void lp_bs_vec_kernel(int op, long fsz, int nrhs, const BsState* __restrict__ S,
                                 float2* __restrict__ p, const float2* __restrict__ r_in,
                                 const float2* __restrict__ v, float2* __restrict__ s,
                                 float2* __restrict__ x, const float2* __restrict__ ph,
                                 const float2* __restrict__ sh, const float2* __restrict__ t,
                                 float2* __restrict__ r_out)
{
    const long n = fsz * nrhs;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const BsState& st = S[i / fsz];
        if (op == 0)
        {
            const float2 pv = p[i], vv = v[i], rv = r_in[i];
            const float2 w = fz(st.omega), b = fz(st.beta);
            const float2 d = make_float2(pv.x - (w.x * vv.x - w.y * vv.y), pv.y - (w.x * vv.y + w.y * vv.x));
            const float2 bd = cmulf(b, d);
            p[i] = make_float2(rv.x + bd.x, rv.y + bd.y);
        }
        else if (op == 1)
        {
            const float2 a = fz(st.alpha), vv = v[i], rv = r_in[i];
            const float2 av = cmulf(a, vv);
            s[i] = make_float2(rv.x - av.x, rv.y - av.y);
        }
        else
        {
            const float2 a = fz(st.alpha), w = fz(st.omega);
            const float2 u1 = cmulf(a, ph[i]), u2 = cmulf(w, sh[i]);
            const float2 xv = x[i];
            x[i] = make_float2(xv.x + u1.x + u2.x, xv.y + u1.y + u2.y);
            const float2 sv = s[i], wt = cmulf(w, t[i]);
            r_out[i] = make_float2(sv.x - wt.x, sv.y - wt.y);
        }
    }
}

// Fused BiCGStab updates with the network's BF16 planar input (4 channels of
// one site per thread; channel c = 2 slice + spin of the operator layout).
// op 0: p = r + beta (p - omega v), planar(p)
// op 1: s = r - alpha v,            planar(s)
__global__ void lp_bs_planar_kernel(int op, int Ls, int V, int planes, int nrhs, const BsState* __restrict__ S,
                                    float2* __restrict__ p, const float2* __restrict__ r,
                                    const float2* __restrict__ v, float2* __restrict__ s,
                                    uint4* __restrict__ planar)
{
    const long fsz = 2L * Ls * V;
    const long n = long(nrhs) * planes * V;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const int h = int(i % V);
        const long q = i / V;
        const int pl = int(q % planes), rhs = int(q / planes);
        const BsState& st = S[rhs];
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            const int sl = 2 * pl + half;  // fifth-dimension slice: channels 2 sl, 2 sl + 1
            if (sl >= Ls)
                continue;
            const long e = long(rhs) * fsz + (long(sl) * V + h) * 2;  // complex index of (slice, site, spin 0)
            const float4 rv = *reinterpret_cast<const float4*>(r + e);
            const float4 vv = *reinterpret_cast<const float4*>(v + e);
            float4 o;
            if (op == 0)
            {
                const float4 pv = *reinterpret_cast<const float4*>(p + e);
                const float2 wo = fz(st.omega), b = fz(st.beta);
                const float2 d0 = make_float2(pv.x - (wo.x * vv.x - wo.y * vv.y), pv.y - (wo.x * vv.y + wo.y * vv.x));
                const float2 d1 = make_float2(pv.z - (wo.x * vv.z - wo.y * vv.w), pv.w - (wo.x * vv.w + wo.y * vv.z));
                const float2 b0 = cmulf(b, d0), b1 = cmulf(b, d1);
                o = make_float4(rv.x + b0.x, rv.y + b0.y, rv.z + b1.x, rv.w + b1.y);
                *reinterpret_cast<float4*>(p + e) = o;
            }
            else
            {
                const float2 al = fz(st.alpha);
                const float2 a0 = cmulf(al, make_float2(vv.x, vv.y)), a1 = cmulf(al, make_float2(vv.z, vv.w));
                o = make_float4(rv.x - a0.x, rv.y - a0.y, rv.z - a1.x, rv.w - a1.y);
                *reinterpret_cast<float4*>(s + e) = o;
            }
            w[2 * half] = pack_bf2(o.x, o.y);
            w[2 * half + 1] = pack_bf2(o.z, o.w);
        }
        planar[(long(rhs) * planes + pl) * V + h] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// x += alpha ph + omega sh ; r = s - omega t ; partials of <rh, r>, <r, r>
// (slots 0, 1) for the next coefficient step.
__global__ void lp_bs_xr_kernel(long fsz, int nblk, const BsState* __restrict__ S, float2* __restrict__ x,
                                const float2* __restrict__ ph, const float2* __restrict__ sh,
                                const float2* __restrict__ s, const float2* __restrict__ t,
                                float2* __restrict__ r, const float2* __restrict__ rh,
                                double2* __restrict__ part)
{
    __shared__ double red[32];
    const int rhs = blockIdx.y;
    const int nrhs = gridDim.y;
    const long ch = (fsz + nblk - 1) / nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < fsz) ? i0 + ch : fsz;
    const long base = long(rhs) * fsz;
    const BsState st = S[rhs];
    const float2 al = fz(st.alpha), wo = fz(st.omega);
    double a_re = 0.0, a_im = 0.0, rr = 0.0;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    {
        const long k = base + i;
        const float2 u1 = cmulf(al, ph[k]), u2 = cmulf(wo, sh[k]);
        const float2 xv = x[k];
        x[k] = make_float2(xv.x + u1.x + u2.x, xv.y + u1.y + u2.y);
        const float2 sv = s[k], wt = cmulf(wo, t[k]);
        const float2 rn = make_float2(sv.x - wt.x, sv.y - wt.y);
        r[k] = rn;
        const float2 hv = rh[k];
        a_re += double(hv.x) * rn.x + double(hv.y) * rn.y;
        a_im += double(hv.x) * rn.y - double(hv.y) * rn.x;
        rr += double(rn.x) * rn.x + double(rn.y) * rn.y;
    }
    a_re = block_sum(a_re, red);
    a_im = block_sum(a_im, red);
    rr = block_sum(rr, red);
    if (threadIdx.x == 0)
    {
        part[(long(0) * nrhs + rhs) * nblk + blockIdx.x] = make_double2(a_re, a_im);
        part[(long(1) * nrhs + rhs) * nblk + blockIdx.x] = make_double2(rr, 0.0);
    }
}

// ---------------------------------------------------------------------------
// flexible GCR (restarted) on the FP32 inner system D e = r
// ---------------------------------------------------------------------------
// Iteration k of a cycle: z_k = N r (network), w_k = D z_k; w_k is
// orthogonalised against w'_0 .. w'_{k-1} of the cycle by classical
// Gram-Schmidt, with every inner product from one pass over the data, into
// w'_k = w_k - sum_i beta_ki w'_i, and the minimal-residual step
// r -= alpha_k w'_k (alpha_k = <w'_k, r> / |w'_k|^2) is taken. The w'_i are
// kept unnormalised with their squared norms. W = W' R with R unit upper
// triangular (R_ik = beta_ki), so the cycle's correction is Z R^-1 alpha,
// formed from the stored network outputs z_k at the end of the cycle: no
// assumption that N is the same operator in every iteration (flexible).
constexpr int kGcrMax = 16;

struct GcrState
{
    double rr;                       // |r|^2 of the inner system
    double nu2[kGcrMax];             // |w'_i|^2 (infinite after a breakdown: w'_i unused)
    double2 beta[kGcrMax][kGcrMax];  // beta[k][i] = <w'_i, w_k> / |w'_i|^2, i < k
    double2 alpha[kGcrMax];
    int active;                      // 1 while iterating
    int iters;
    int breakdown;                   // steps skipped because w_k lay in the span of the w'_i
    unsigned cnt;                    // blocks of the current pass that are done
};

struct GcrArgs
{
    long f4;            // float4 (two complex numbers) per right-hand side
    long slot4;         // float4 per stored vector of all right-hand sides
    int nblk;           // blocks per right-hand side
    float4* W;          // w'_0 .. w'_{m-1}: [slot][rhs][f4]
    const float4* Z;    // z_0 .. z_{m-1}
    float4* r;
    float4* x;
    uint4* planar;      // BF16 planar copy of r for the network (null: not kept)
    int Ls, V, planes;
    GcrState* S;
    int* flags;         // [0, nrhs): active, [nrhs, 2 nrhs): iterations
    double* part;       // [rhs][blk][64]
    double tgt2;
    int maxit;
};

__device__ __forceinline__ float warp_sum_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Whether this block is the last of its right-hand side's nblk blocks to
// finish the pass (its partials are then all visible to it).
__device__ __forceinline__ bool gcr_last_block(GcrState* st, int nblk, bool* flag)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        *flag = atomicAdd(&st->cnt, 1u) == unsigned(nblk - 1);
    __syncthreads();
    if (!*flag)
        return false;
    __threadfence();
    return true;
}

// Pass A of iteration k = NV: <w_k, w_k>, <w_k, r> and, for i < k,
// <w'_i, w_k>, <w'_i, r>; the last block forms beta_k*, |w'_k|^2 and alpha_k.
template <int NV>
__global__ void __launch_bounds__(256) lp_gcr_dots_kernel(GcrArgs g)
{
    constexpr int NVAL = 3 + 4 * NV;
    __shared__ double sred[8][NVAL];
    __shared__ double tot[NVAL];
    // launched as a programmatic dependent: the previous kernel's results first
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __shared__ bool last;
    const int rhs = blockIdx.y;
    const long ch = (g.f4 + g.nblk - 1) / g.nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < g.f4) ? i0 + ch : g.f4;
    const long base = long(rhs) * g.f4;
    const float4* __restrict__ w = g.W + NV * g.slot4 + base;
    const float4* __restrict__ r = g.r + base;
    float acc[NVAL];
#pragma unroll
    for (int v = 0; v < NVAL; ++v)
        acc[v] = 0.f;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    {
        const float4 a = w[i], b = r[i];
        acc[0] += a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w;
        acc[1] += a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
        acc[2] += a.x * b.y - a.y * b.x + a.z * b.w - a.w * b.z;
#pragma unroll
        for (int j = 0; j < NV; ++j)
        {
            const float4 q = g.W[j * g.slot4 + base + i];
            acc[3 + 4 * j] += q.x * a.x + q.y * a.y + q.z * a.z + q.w * a.w;
            acc[4 + 4 * j] += q.x * a.y - q.y * a.x + q.z * a.w - q.w * a.z;
            acc[5 + 4 * j] += q.x * b.x + q.y * b.y + q.z * b.z + q.w * b.w;
            acc[6 + 4 * j] += q.x * b.y - q.y * b.x + q.z * b.w - q.w * b.z;
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NVAL; ++v)
    {
        const float s = warp_sum_f(acc[v]);
        if (lane == 0)
            sred[wid][v] = s;
    }
    __syncthreads();
    double* part = g.part + (long(rhs) * g.nblk + blockIdx.x) * 64;
    for (int v = threadIdx.x; v < NVAL; v += blockDim.x)
    {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
            s += sred[q][v];
        part[v] = s;
    }
    GcrState* st = g.S + rhs;
    if (!gcr_last_block(st, g.nblk, &last))
        return;
    for (int v = threadIdx.x; v < NVAL; v += blockDim.x)
    {
        double s = 0.0;
        for (int b = 0; b < g.nblk; ++b)
            s += __ldcg(g.part + (long(rhs) * g.nblk + b) * 64 + v);
        tot[v] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    st->cnt = 0u;
    const int k = NV;
    bool skip = !st->active;
    double nu2 = tot[0];
    double2 num = make_double2(tot[1], tot[2]);
    for (int i = 0; i < k; ++i)
    {
        const double2 gw = make_double2(tot[3 + 4 * i], tot[4 + 4 * i]);
        const double2 gr = make_double2(tot[5 + 4 * i], tot[6 + 4 * i]);
        const double ni = st->nu2[i];
        const double2 b = isfinite(ni) ? make_double2(gw.x / ni, gw.y / ni) : make_double2(0.0, 0.0);
        st->beta[k][i] = b;
        nu2 -= isfinite(ni) ? (gw.x * gw.x + gw.y * gw.y) / ni : 0.0;
        // <w'_k, r> = <w_k, r> - sum_i conj(beta_ki) <w'_i, r>
        num.x -= b.x * gr.x + b.y * gr.y;
        num.y -= b.x * gr.y - b.y * gr.x;
    }
    const bool bad = !(nu2 > 1e-10 * tot[0]) || !isfinite(nu2) || !zfinite(num);
    if (!skip && bad)
        st->breakdown += 1;
    if (skip || bad)
    {
        for (int i = 0; i < k; ++i)
            st->beta[k][i] = make_double2(0.0, 0.0);
        st->nu2[k] = INFINITY;
        st->alpha[k] = make_double2(0.0, 0.0);
        return;
    }
    st->nu2[k] = nu2;
    st->alpha[k] = make_double2(num.x / nu2, num.y / nu2);
}

// Pass B of iteration k = NV: w'_k = w_k - sum_i beta_ki w'_i (stored over
// w_k), r -= alpha_k w'_k, the BF16 planar copy of r (thread per plane and
// site) and |r|^2; the last block updates the stopping state.
template <int NV>
__global__ void __launch_bounds__(256) lp_gcr_update_kernel(GcrArgs g)
{
    __shared__ float2 cb[NV + 1];  // beta_k0 .. beta_k(k-1), alpha_k
    __shared__ double red[32];
    __shared__ bool last;
    asm volatile("griddepcontrol.wait;" ::: "memory");  // as lp_gcr_dots_kernel
    const int rhs = blockIdx.y, nrhs = gridDim.y;
    GcrState* st = g.S + rhs;
    if (int(threadIdx.x) <= NV)
    {
        const double2 c = int(threadIdx.x) < NV ? st->beta[NV][threadIdx.x] : st->alpha[NV];
        cb[threadIdx.x] = make_float2(float(c.x), float(c.y));
    }
    __syncthreads();
    const long items = long(g.planes) * g.V;
    const long ch = (items + g.nblk - 1) / g.nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < items) ? i0 + ch : items;
    const long base = long(rhs) * g.f4;
    float4* __restrict__ w = g.W + NV * g.slot4 + base;
    float4* __restrict__ r = g.r + base;
    const float2 al = cb[NV];
    double rr = 0.0;
    for (long it = i0 + threadIdx.x; it < i1; it += blockDim.x)
    {
        const int h = int(it % g.V), pl = int(it / g.V);
        uint32_t pk[4] = {0u, 0u, 0u, 0u};
        float racc = 0.f;
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            const int sl = 2 * pl + half;
            if (sl >= g.Ls)
                continue;
            const long e = long(sl) * g.V + h;  // float4 of (slice, site): both spins
            float4 a = w[e];
#pragma unroll
            for (int j = 0; j < NV; ++j)
            {
                const float4 q = g.W[j * g.slot4 + base + e];
                const float2 b = cb[j];
                a.x -= b.x * q.x - b.y * q.y;
                a.y -= b.x * q.y + b.y * q.x;
                a.z -= b.x * q.z - b.y * q.w;
                a.w -= b.x * q.w + b.y * q.z;
            }
            if (NV > 0)
                w[e] = a;
            float4 rv = r[e];
            rv.x -= al.x * a.x - al.y * a.y;
            rv.y -= al.x * a.y + al.y * a.x;
            rv.z -= al.x * a.z - al.y * a.w;
            rv.w -= al.x * a.w + al.y * a.z;
            r[e] = rv;
            racc += rv.x * rv.x + rv.y * rv.y + rv.z * rv.z + rv.w * rv.w;
            pk[2 * half] = pack_bf2(rv.x, rv.y);
            pk[2 * half + 1] = pack_bf2(rv.z, rv.w);
        }
        rr += racc;
        if (g.planar)
            g.planar[(long(rhs) * g.planes + pl) * g.V + h] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
    rr = block_sum(rr, red);
    if (threadIdx.x == 0)
        g.part[(long(rhs) * g.nblk + blockIdx.x) * 64] = rr;
    if (!gcr_last_block(st, g.nblk, &last))
        return;
    if (threadIdx.x != 0)
        return;
    double s = 0.0;
    for (int b = 0; b < g.nblk; ++b)
        s += __ldcg(g.part + (long(rhs) * g.nblk + b) * 64);
    st->cnt = 0u;
    st->rr = s;
    if (st->active)
    {
        st->iters += 1;
        st->active = (s > g.tgt2 && st->iters < g.maxit && isfinite(s)) ? 1 : 0;
    }
    g.flags[rhs] = st->active;
    g.flags[nrhs + rhs] = st->iters;
}

// End of a cycle of m iterations: x += Z R^-1 alpha (gamma by back
// substitution, gamma_k = alpha_k - sum_{j>k} beta_jk gamma_j).
__global__ void __launch_bounds__(256) lp_gcr_x_kernel(GcrArgs g, int m)
{
    __shared__ float2 gam[kGcrMax];
    asm volatile("griddepcontrol.wait;" ::: "memory");  // as lp_gcr_dots_kernel
    const int rhs = blockIdx.y;
    const GcrState* st = g.S + rhs;
    if (threadIdx.x == 0)
    {
        double2 gm[kGcrMax];
        for (int k = m - 1; k >= 0; --k)
        {
            double2 v = st->alpha[k];
            for (int j = k + 1; j < m; ++j)
            {
                const double2 b = st->beta[j][k];
                v.x -= b.x * gm[j].x - b.y * gm[j].y;
                v.y -= b.x * gm[j].y + b.y * gm[j].x;
            }
            gm[k] = v;
            gam[k] = make_float2(float(v.x), float(v.y));
        }
    }
    __syncthreads();
    const long ch = (g.f4 + g.nblk - 1) / g.nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < g.f4) ? i0 + ch : g.f4;
    const long base = long(rhs) * g.f4;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    {
        float4 xv = g.x[base + i];
        for (int j = 0; j < m; ++j)
        {
            const float4 q = g.Z[j * g.slot4 + base + i];
            const float2 c = gam[j];
            xv.x += c.x * q.x - c.y * q.y;
            xv.y += c.x * q.y + c.y * q.x;
            xv.z += c.x * q.z - c.y * q.w;
            xv.w += c.x * q.w + c.y * q.z;
        }
        g.x[base + i] = xv;
    }
}

// Start of an inner solve: |r|^2 from the partials of lp_dots_kernel (slot
// 0), active where the host asked and |r|^2 > tgt2.
__global__ void lp_gcr_init_kernel(const double2* __restrict__ part, int nrhs, int nblk, GcrState* __restrict__ S,
                                   const int* __restrict__ want, int* __restrict__ flags, double tgt2)
{
    const int rhs = blockIdx.x * blockDim.x + threadIdx.x;
    if (rhs >= nrhs)
        return;
    GcrState& st = S[rhs];
    st.rr = sum_part(part, 0, nrhs, rhs, nblk).x;
    st.active = (want[rhs] && st.rr > tgt2) ? 1 : 0;
    st.iters = 0;
    st.breakdown = 0;
    st.cnt = 0u;
    flags[rhs] = st.active;
    flags[nrhs + rhs] = 0;
}

// Outer (FP64) steps.
// r = b - Ax (tmp holds A x), partial |r|^2 into part (slot 0).
__global__ void lp_resid_kernel(const double2* __restrict__ b, const double2* __restrict__ Ax,
                                double2* __restrict__ r, long fsz, int nblk, double* __restrict__ part)
{
    __shared__ double red[32];
    const int rhs = blockIdx.y;
    const long ch = (fsz + nblk - 1) / nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < fsz) ? i0 + ch : fsz;
    double s = 0.0;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    {
        const long k = long(rhs) * fsz + i;
        const double2 v = make_double2(b[k].x - Ax[k].x, b[k].y - Ax[k].y);
        r[k] = v;
        s += v.x * v.x + v.y * v.y;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0)
        part[long(rhs) * nblk + blockIdx.x] = s;
}

__global__ void lp_norm_kernel(const double2* __restrict__ a, long fsz, int nblk, double* __restrict__ part)
{
    __shared__ double red[32];
    const int rhs = blockIdx.y;
    const long ch = (fsz + nblk - 1) / nblk;
    const long i0 = blockIdx.x * ch, i1 = (i0 + ch < fsz) ? i0 + ch : fsz;
    double s = 0.0;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    {
        const double2 v = a[long(rhs) * fsz + i];
        s += v.x * v.x + v.y * v.y;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0)
        part[long(rhs) * nblk + blockIdx.x] = s;
}

__global__ void lp_sum_kernel(const double* __restrict__ part, int nrhs, int nblk, double* __restrict__ out)
{
    const int rhs = blockIdx.x * blockDim.x + threadIdx.x;
    if (rhs >= nrhs)
        return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b)
        s += part[long(rhs) * nblk + b];
    out[rhs] = s;
}

// r32 = r64 * inv[rhs] (inv = 0 leaves a zero field)
__global__ void lp_down_kernel(const double2* __restrict__ r, const double* __restrict__ inv, long fsz,
                               int nrhs, float2* __restrict__ r32)
{
    const long n = fsz * nrhs;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const double s = inv[i / fsz];
        r32[i] = make_float2(float(r[i].x * s), float(r[i].y * s));
    }
}

// x += scale[rhs] * e32
__global__ void lp_up_kernel(double2* __restrict__ x, const float2* __restrict__ e, const double* __restrict__ scale,
                             long fsz, int nrhs)
{
    const long n = fsz * nrhs;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
    {
        const double s = scale[i / fsz];
        if (s != 0.0)
            x[i] = make_double2(x[i].x + s * e[i].x, x[i].y + s * e[i].y);
    }
}

__global__ void lp_f64_to_f32_kernel(const double2* __restrict__ a, float2* __restrict__ b, long n)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        b[i] = make_float2(float(a[i].x), float(a[i].y));
}

// e = x* - x_k (FP32)
__global__ void lp_diff_kernel(const double2* __restrict__ a, const double2* __restrict__ b,
                               float2* __restrict__ out, long n)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        out[i] = make_float2(float(a[i].x - b[i].x), float(a[i].y - b[i].y));
}

}  // namespace dwfb

// ===========================================================================
// host side
// ===========================================================================
struct LpNet
{
    int C0 = 0, H = 0;
    int cin[kLpLayers], cout[kLpLayers], ntf[kLpLayers], nta[kLpLayers];
    long woff[kLpLayers + 1];          // complex offsets of each layer's weights
    long bf_off[kLpLayers + 1];        // uint2 offsets of forward fragments
    long ba_off[kLpLayers + 1];        // and of adjoint fragments
    float2* W = nullptr;               // FP32 master weights
    float2* G = nullptr;               // gradient
    float* m = nullptr;                // Adam moments (2 floats per complex weight)
    float* v = nullptr;
    long adam_t = 0;
    uint2* Bf = nullptr;
    uint2* Ba = nullptr;
    // tcgen05 B operands (forward and adjoint) and their real column counts
    uint4* Btf = nullptr;
    uint4* Bta = nullptr;
    long tf_off[kLpLayers + 1], ta_off[kLpLayers + 1];
    int ncf[kLpLayers], nca[kLpLayers];
    int variant = -1;                  // -1 auto, 0 mma.sync kernel, 1 tcgen05 kernel
    int auto_variant = -1;             // the automatic choice in force (-1: tcgen05 where it fits)
    std::map<int, int> auto_tuned;     // automatic choice per batch-size bucket
    std::map<long, int> conv_bps;      // resident blocks per SM of the mma.sync kernel (nt, smem)
    bool smem_set = false;             // layer kernels' shared-memory limit raised on this device
    int* err_d = nullptr;              // bounded-wait error flag of the tcgen05 kernel
    float2* T = nullptr;               // transports [nconf][V][9]
    int T_cap = 0;
    uint64_t T_version = ~0ull;
    // activations: layer inputs of the last forward pass (training)
    int act_rhs = 0;
    float2* act[kLpLayers] = {nullptr, nullptr, nullptr, nullptr};
    float2* hid[2] = {nullptr, nullptr};
    uint4* hb[2] = {nullptr, nullptr};  // BF16 planar hidden fields (tcgen05 chain)
    float2* gbuf[2] = {nullptr, nullptr};   // gradients flowing back (operator and hidden layout)
    float2* gpart = nullptr;
    size_t gpart_cap = 0;
    int grad_blocks = 0;
    double* lpart = nullptr;
    double* lscale = nullptr;
    double* dloss = nullptr;
    size_t lpart_cap = 0;
    int* dconf = nullptr;
    int dconf_cap = 0;
    // training pairs (FP32, operator layout)
    int npairs = 0;
    float2* pr_rho = nullptr;
    float2* pr_e = nullptr;
    std::vector<int> pr_conf;
    // flexible GCR workspace: m stored network outputs z and orthogonalised w'
    float2* g_Z = nullptr;
    float2* g_W = nullptr;
    size_t g_cap = 0;                   // complex numbers of each
    GcrState* g_state = nullptr;
    int* g_flags = nullptr;             // [3][nrhs]: active, iterations, wanted
    double* g_part = nullptr;
    int g_rhs = 0;
    // captured chunks of four GCR iterations, per first iteration k0 / 4
    cudaGraphExec_t gcr_exec[kGcrMax / 4] = {};
    std::vector<uintptr_t> gcr_key[kGcrMax / 4];
    size_t gcr_nodes[kGcrMax / 4] = {};
    // solver workspace
    int s_rhs = 0;
    float2* s_f32[9] = {};      // r, rh, p, v, s, t, ph, sh, x
    double2* s_r64 = nullptr;
    double2* s_t64 = nullptr;
    double2* s_rhs64 = nullptr;
    double2* s_part2 = nullptr;
    double* s_part = nullptr;
    double* s_val = nullptr;    // per-rhs scalars [4][nrhs]
    BsState* s_state = nullptr;
    // captured inner iterations of the solve (replayed per chunk) and its key
    cudaGraphExec_t g_exec = nullptr;
    std::vector<uintptr_t> g_key;
    size_t g_nodes = 0;
    // solver settings
    int krylov = 0;                     // 0 flexible GCR, 1 BiCGStab
    // GCR restart length (4, 8, 12 or 16): at 64x64x16 with 28 sources and
    // inner_tol 3e-4, 4 / 8 / 12 / 16 gave 800 / 740 / 667 / 608 solves/s
    // (BiCGStab: 563); the orthogonalisation passes grow with the restart
    // length faster than the iterations fall (133 / 122 / 118 / 117)
    int gcr_m = 4;
    // inner_tol 1e-3 / 3e-4 / 1e-4 -> 685 / 800 / 707 solves/s (GCR(4), as above)
    double inner_tol = 3e-4;
    int inner_max = 400;
    int outer_max = 40;
    long iters_total = 0;
};

namespace dwfb {
namespace {

template <typename T>
int lp_grow(dwf_ctx* c, T*& p, size_t n)
{
    if (p)
        cudaFree(p);
    p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    return DWF_OK;
}

// Output column tiles of the mma.sync layer (8 real columns each) and real
// output columns of the tcgen05 layer, rounded up to the instantiated kernel
// shapes (the padded columns hold zero weights and are not stored).
int nt_of(int cout)
{
    const int n = (2 * cout + 7) / 8;
    return n <= 2 ? n : (n <= 4 ? 4 : (n <= 6 ? 6 : (n <= 8 ? 8 : 12)));
}

int ncol_of(int cout)
{
    const int n = (2 * cout + 15) / 16 * 16;
    return n <= 64 ? n : 96;
}

int grid_for(long n, int nsm) { return int(std::max<long>(1, std::min<long>((n + 255) / 256, 8L * nsm))); }

int cpad_of(int c) { return (c + 7) / 8 * 8; }

int set_conv_smem(dwf_ctx* c)
{
    // per context (each context drives one device); the attribute is per device
    if (c->lp->smem_set)
        return DWF_OK;
    const int mx = 220 * 1024;
    CK(cudaFuncSetAttribute(lp_conv_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_conv_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_conv_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_conv_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_conv_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_conv_kernel<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_tc_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_tc_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    CK(cudaFuncSetAttribute(lp_tc_kernel<96>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    c->lp->smem_set = true;
    return DWF_OK;
}

// Pack the BF16 fragments of every layer (forward and adjoint) from W.
int lp_pack(dwf_ctx* c)
{
    LpNet* n = c->lp;
    for (int l = 0; l < kLpLayers; ++l)
    {
        const long nf = n->bf_off[l + 1] - n->bf_off[l];
        const long na = n->ba_off[l + 1] - n->ba_off[l];
        lp_pack_kernel<<<grid_for(nf, c->nsm), 256, 0, c->stream>>>(
            n->W + n->woff[l], n->cin[l], n->cout[l], 0, cpad_of(n->cin[l]), n->ntf[l],
            n->Bf + n->bf_off[l]);
        // adjoint layer: cin' = cout, cout' = cin
        lp_pack_kernel<<<grid_for(na, c->nsm), 256, 0, c->stream>>>(
            n->W + n->woff[l], n->cin[l], n->cout[l], 1, cpad_of(n->cout[l]), n->nta[l],
            n->Ba + n->ba_off[l]);
        const long tf = (n->tf_off[l + 1] - n->tf_off[l]) * 8;
        const long ta = (n->ta_off[l + 1] - n->ta_off[l]) * 8;
        lp_pack_tc_kernel<<<grid_for(tf, c->nsm), 256, 0, c->stream>>>(
            n->W + n->woff[l], n->cin[l], n->cout[l], 0, cpad_of(n->cin[l]), n->ncf[l],
            reinterpret_cast<__nv_bfloat16*>(n->Btf + n->tf_off[l]));
        lp_pack_tc_kernel<<<grid_for(ta, c->nsm), 256, 0, c->stream>>>(
            n->W + n->woff[l], n->cin[l], n->cout[l], 1, cpad_of(n->cout[l]), n->nca[l],
            reinterpret_cast<__nv_bfloat16*>(n->Bta + n->ta_off[l]));
        c->launches += 4;
    }
    CK(cudaGetLastError());
    return DWF_OK;
}

int lp_transports(dwf_ctx* c)
{
    LpNet* n = c->lp;
    if (n->T_version == c->gauge_version && n->T_cap >= c->nconf)
        return DWF_OK;
    if (n->T_cap < c->nconf)
    {
        ST(lp_grow(c, n->T, size_t(c->nconf) * c->L.V * 9));
        n->T_cap = c->nconf;
    }
    lp_transport_kernel<<<grid_for(long(c->nconf) * c->L.V, c->nsm), 256, 0, c->stream>>>(
        c->L, c->U64, c->usz(), c->nconf, n->T);
    c->launches += 1;
    CK(cudaGetLastError());
    n->T_version = c->gauge_version;
    return DWF_OK;
}

int lp_conf(dwf_ctx* c, int nrhs, const int* conf_h, const int** conf_d)
{
    LpNet* n = c->lp;
    if (nrhs > n->dconf_cap)
    {
        ST(lp_grow(c, n->dconf, nrhs));
        n->dconf_cap = nrhs;
    }
    std::vector<int> cf(nrhs, 0);
    if (conf_h)
        std::copy(conf_h, conf_h + nrhs, cf.begin());
    for (int k = 0; k < nrhs; ++k)
        if (cf[k] < 0 || cf[k] >= c->nconf)
            return ctx_fail(c, DWF_BAD_ARG, "learned: configuration index out of range");
    CK(cudaMemcpyAsync(n->dconf, cf.data(), nrhs * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    *conf_d = n->dconf;
    return DWF_OK;
}

FieldLayout op_layout(const dwf_ctx* c)
{
    // operator layout: channel c = 2 s + spin; a Wilson field is the Ls = 1 case
    return FieldLayout{c->fsz(), 2, 2, 2 * c->L.V};
}

FieldLayout net_layout(const dwf_ctx* c, int C) { return FieldLayout{long(c->L.V) * C, C, C, 0}; }

// The layer kernel choice in force: the explicit setting, else the automatic one.
int lp_eff_variant(const LpNet* n) { return n->variant >= 0 ? n->variant : n->auto_variant; }

// Whether the tcgen05 kernel (and its BF16 planar chain) may run: chosen
// explicitly, or automatic before any timing.
bool lp_tc_allowed(const LpNet* n)
{
    const int v = lp_eff_variant(n);
    return v == 1 || v == -1;
}

// Whether the tcgen05 kernel takes layer l (its shared-memory tile fits).
bool tc_fits(const dwf_ctx* c, int l, bool adjoint)
{
    const LpNet* n = c->lp;
    const int ci = adjoint ? n->cout[l] : n->cin[l];
    const int co = adjoint ? n->cin[l] : n->cout[l];
    const int ncol = ncol_of(co);
    return ncol <= 96 && tc_smem_bytes(cpad_of(ci), ncol, c->L.Nx, 1) <= size_t(220 * 1024);
}

// One layer (forward or adjoint) on device fields. in_bf / out_bf (tcgen05
// kernel only): BF16 planar input / output in place of in / out.
int lp_layer(dwf_ctx* c, int l, bool adjoint, int nrhs, const int* conf_d, const float2* in,
             FieldLayout li, float2* out, FieldLayout lo, const uint4* in_bf = nullptr,
             uint4* out_bf = nullptr)
{
    LpNet* n = c->lp;
    const int ci = adjoint ? n->cout[l] : n->cin[l];
    const int co = adjoint ? n->cin[l] : n->cout[l];
    const int ncol = ncol_of(co);
    // two CTAs per SM (one window buffer each) where their shared memory and
    // TMEM fit, else one double-buffered CTA
    const bool two = 2 * tc_smem_bytes(cpad_of(ci), ncol, c->L.Nx, 1) <= size_t(226 * 1024) &&
                     2 * tc_tmem_cols(ncol) <= 512u;
    // one CTA double-buffers its window where the second buffer still fits
    const int nbuf = (two || tc_smem_bytes(cpad_of(ci), ncol, c->L.Nx, 2) > size_t(220 * 1024)) ? 1 : 2;
    const size_t tsm = tc_smem_bytes(cpad_of(ci), ncol, c->L.Nx, nbuf);
    const bool tc_ok = tc_fits(c, l, adjoint);
    if (lp_tc_allowed(n) && tc_ok)
    {
        TcArgs t;
        t.in = in;
        t.out = out;
        t.li = li;
        t.lo = lo;
        t.cin = ci;
        t.cout = co;
        t.cpad = cpad_of(ci);
        t.ncol = ncol;
        t.B = adjoint ? n->Bta + n->ta_off[l] : n->Btf + n->tf_off[l];
        t.T = n->T;
        t.conf = conf_d;
        t.conf0 = 0;
        t.Nt = c->L.Nt;
        t.Nx = c->L.Nx;
        t.V = c->L.V;
        t.nrhs = nrhs;
        t.err = n->err_d;
        t.timeout_ns = c->timeout_ns;
        t.in_bf = in_bf;
        t.out_bf = out_bf;
        t.nbuf = nbuf;
        const long ntiles = tc_tiles_per_rhs(c->L.Nt, c->L.Nx) * nrhs;
        const int grid = int(std::max<long>(1, std::min<long>(ntiles, long(two ? 2 : 1) * c->nsm)));
        ST(set_conv_smem(c));
        // programmatic dependent launch (the kernel waits for its predecessor
        // before touching any field; see lp_tc_kernel)
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = DWFB_TC_PDL;
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kTcThreads);
        cfg.dynamicSmemBytes = tsm;
        cfg.stream = c->stream;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        switch (ncol)
        {
        case 16: CK(cudaLaunchKernelEx(&cfg, lp_tc_kernel<16>, t)); break;
        case 32: CK(cudaLaunchKernelEx(&cfg, lp_tc_kernel<32>, t)); break;
        case 48: CK(cudaLaunchKernelEx(&cfg, lp_tc_kernel<48>, t)); break;
        case 64: CK(cudaLaunchKernelEx(&cfg, lp_tc_kernel<64>, t)); break;
        case 96: CK(cudaLaunchKernelEx(&cfg, lp_tc_kernel<96>, t)); break;
        default: return ctx_fail(c, DWF_BAD_ARG, "learned: unsupported channel count");
        }
        c->launches += 1;
        CK(cudaGetLastError());
        return DWF_OK;
    }
    if (n->variant == 1 || in_bf || out_bf)
        return ctx_fail(c, DWF_BAD_ARG, "learned: the tcgen05 layer does not fit this lattice / width");
    ConvArgs a;
    a.in = in;
    a.out = out;
    a.li = li;
    a.lo = lo;
    a.cin = adjoint ? n->cout[l] : n->cin[l];
    a.cout = adjoint ? n->cin[l] : n->cout[l];
    a.cpad = cpad_of(a.cin);
    a.tx = std::min(64, (c->L.Nx + 15) / 16 * 16);
    a.B = adjoint ? n->Ba + n->ba_off[l] : n->Bf + n->bf_off[l];
    a.T = n->T;
    a.conf = conf_d;
    a.conf0 = 0;
    a.Nt = c->L.Nt;
    a.Nx = c->L.Nx;
    a.V = c->L.V;
    a.nrhs = nrhs;
    const int nt = nt_of(a.cout);
    const size_t smem = conv_smem_bytes(a.cpad, nt, a.tx);
    const long ntiles = long((a.Nt + kTileRows - 1) / kTileRows) * ((a.Nx + a.tx - 1) / a.tx) * nrhs;
    ST(set_conv_smem(c));
    const void* fn = nullptr;
    switch (nt)
    {
    case 1: fn = reinterpret_cast<const void*>(&lp_conv_kernel<1>); break;
    case 2: fn = reinterpret_cast<const void*>(&lp_conv_kernel<2>); break;
    case 4: fn = reinterpret_cast<const void*>(&lp_conv_kernel<4>); break;
    case 6: fn = reinterpret_cast<const void*>(&lp_conv_kernel<6>); break;
    case 8: fn = reinterpret_cast<const void*>(&lp_conv_kernel<8>); break;
    case 12: fn = reinterpret_cast<const void*>(&lp_conv_kernel<12>); break;
    default: return ctx_fail(c, DWF_BAD_ARG, "learned: unsupported channel count");
    }
    // every block walks tiles in turn (stage, MMAs, transporters, store), so
    // the tiles in flight per SM are the resident blocks: fill them all
    const long key = long(nt) * (1L << 32) + long(smem);
    auto it = n->conv_bps.find(key);
    if (it == n->conv_bps.end())
    {
        int bps = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, kConvWarps * 32, smem));
        it = n->conv_bps.emplace(key, std::max(1, bps)).first;
    }
    const int grid = int(std::max<long>(1, std::min<long>(ntiles, long(it->second) * c->nsm)));
    void* args[] = {&a};
    CK(cudaLaunchKernel(fn, dim3(grid), dim3(kConvWarps * 32), args, smem, c->stream));
    c->launches += 1;
    CK(cudaGetLastError());
    return DWF_OK;
}

int lp_ensure_act(dwf_ctx* c, int nrhs)
{
    LpNet* n = c->lp;
    if (nrhs <= n->act_rhs)
        return DWF_OK;
    const size_t hid = size_t(nrhs) * c->L.V * n->H;
    const size_t op = size_t(nrhs) * c->fsz();
    for (int l = 1; l < kLpLayers; ++l)
        ST(lp_grow(c, n->act[l], hid));
    ST(lp_grow(c, n->hid[0], std::max(hid, op)));
    ST(lp_grow(c, n->hid[1], std::max(hid, op)));
    ST(lp_grow(c, n->gbuf[0], std::max(hid, op)));
    ST(lp_grow(c, n->gbuf[1], std::max(hid, op)));
    const size_t pl = size_t(std::max(cpad_of(n->C0), cpad_of(n->H)) / 4);
    ST(lp_grow(c, n->hb[0], size_t(nrhs) * pl * c->L.V));
    ST(lp_grow(c, n->hb[1], size_t(nrhs) * pl * c->L.V));
    n->act_rhs = nrhs;
    return DWF_OK;
}

// out = N in (adjoint: N^dag in), operator layout, FP32. Hidden fields in
// hid[0], hid[1]; with `keep`, the layer inputs are also kept in act[] (act[0]
// is `in` itself).
int lp_net(dwf_ctx* c, bool adjoint, int nrhs, const int* conf_d, const float2* in, float2* out,
           bool keep, bool planar_ready = false)
{
    LpNet* n = c->lp;
    ST(lp_ensure_act(c, nrhs));
    const FieldLayout lop = op_layout(c), lh = net_layout(c, n->H);
    bool chain = !keep && lp_tc_allowed(n);
    for (int l = 0; l < kLpLayers; ++l)
        chain = chain && tc_fits(c, l, adjoint);
    if (chain)
    {
        // tcgen05 chain: BF16 planar activations between the layers
        const int l0 = adjoint ? kLpLayers - 1 : 0;
        const int cin0 = adjoint ? n->cout[l0] : n->cin[l0];
        const int planes0 = cpad_of(cin0) / 4;
        const long np = long(nrhs) * planes0 * c->L.V;
        if (!planar_ready)
        {
            lp_to_planar_kernel<<<grid_for(np, c->nsm), 256, 0, c->stream>>>(in, lop, cin0, planes0, c->L.V,
                                                                              nrhs, n->hb[0]);
            c->launches += 1;
        }
        for (int s = 0; s < kLpLayers; ++s)
        {
            const int l = adjoint ? kLpLayers - 1 - s : s;
            const bool last = (s == kLpLayers - 1);
            ST(lp_layer(c, l, adjoint, nrhs, conf_d, nullptr, lop, last ? out : nullptr, lop, n->hb[s & 1],
                        last ? nullptr : n->hb[(s + 1) & 1]));
        }
        return DWF_OK;
    }
    const float2* cur = in;
    FieldLayout lcur = lop;
    for (int s = 0; s < kLpLayers; ++s)
    {
        const int l = adjoint ? kLpLayers - 1 - s : s;
        const bool last = (s == kLpLayers - 1);
        float2* dst = last ? out : (keep ? n->act[s + 1] : n->hid[s & 1]);
        if (keep)
            n->act[0] = const_cast<float2*>(in);
        ST(lp_layer(c, l, adjoint, nrhs, conf_d, cur, lcur, dst, last ? lop : lh));
        cur = dst;
        lcur = lh;
    }
    return DWF_OK;
}

// Whether lp_net runs the tcgen05 chain with BF16 planar activations.
bool lp_chain(const dwf_ctx* c, bool adjoint)
{
    bool chain = lp_tc_allowed(c->lp);
    for (int l = 0; l < kLpLayers; ++l)
        chain = chain && tc_fits(c, l, adjoint);
    return chain;
}

int lp_ensure_lpart(dwf_ctx* c, size_t n)
{
    LpNet* L = c->lp;
    if (n <= L->lpart_cap)
        return DWF_OK;
    ST(lp_grow(c, L->lpart, n));
    L->lpart_cap = n;
    return DWF_OK;
}

// Loss of the current network on pairs (rho, e) (device, operator layout),
// the gradient into n->G. loss_out: host (may be null: stays on device).
int lp_loss_grad(dwf_ctx* c, int nrhs, const int* conf_d, const float2* rho, const float2* e,
                 double* loss_out)
{
    LpNet* n = c->lp;
    ST(lp_ensure_act(c, nrhs));
    const long fs = c->fsz();
    // forward, keeping the layer inputs; output into gbuf[1]
    float2* out = n->gbuf[1];
    ST(lp_net(c, false, nrhs, conf_d, rho, out, true));
    const int nblk = int(std::min<long>(64, (fs + 4095) / 4096));
    ST(lp_ensure_lpart(c, size_t(nrhs) * nblk * 2));
    if (!n->lscale)
        ST(lp_grow(c, n->lscale, 65536));
    if (!n->dloss)
        ST(lp_grow(c, n->dloss, 1));
    lp_loss_partials_kernel<<<dim3(nblk, nrhs), 256, 0, c->stream>>>(out, e, fs, nblk, n->lpart);
    lp_loss_finish_kernel<<<1, 256, 0, c->stream>>>(n->lpart, nrhs, nblk, n->lscale, n->dloss);
    float2* g = n->gbuf[0];
    lp_loss_grad_kernel<<<grid_for(fs * nrhs, c->nsm), 256, 0, c->stream>>>(out, e, fs, nrhs, n->lscale, g);
    c->launches += 3;
    CK(cudaGetLastError());
    // backward through the layers
    const FieldLayout lop = op_layout(c), lh = net_layout(c, n->H);
    const float2* gcur = g;
    FieldLayout lg = lop;
    const int nblk_g = std::max(1, std::min(2 * c->nsm, (c->L.V * nrhs + kGradSites - 1) / kGradSites));
    long gmax = 0;
    for (int l = 0; l < kLpLayers; ++l)
        gmax = std::max<long>(gmax, 9L * n->cin[l] * n->cout[l]);
    if (size_t(nblk_g) * gmax > n->gpart_cap)
    {
        ST(lp_grow(c, n->gpart, size_t(nblk_g) * gmax));
        n->gpart_cap = size_t(nblk_g) * gmax;
    }
    for (int l = kLpLayers - 1; l >= 0; --l)
    {
        GradArgs a;
        a.in = n->act[l];
        a.g = gcur;
        a.li = (l == 0) ? lop : lh;
        a.lg = lg;
        a.cin = n->cin[l];
        a.cout = n->cout[l];
        a.T = n->T;
        a.conf = conf_d;
        a.conf0 = 0;
        a.Nt = c->L.Nt;
        a.Nx = c->L.Nx;
        a.V = c->L.V;
        a.nrhs = nrhs;
        a.part = n->gpart;
        const size_t smem = size_t(kGradSites) * (a.cin + a.cout) * sizeof(float2);
        if (a.cin * a.cout <= kGradThreads * 4)
            lp_wgrad_kernel<4><<<nblk_g, kGradThreads, smem, c->stream>>>(a);
        else
            lp_wgrad_kernel<kGradMaxPer><<<nblk_g, kGradThreads, smem, c->stream>>>(a);
        const int E = 9 * a.cin * a.cout;
        lp_grad_reduce_kernel<<<(E + 255) / 256, 256, 0, c->stream>>>(n->gpart, nblk_g, E, n->G + n->woff[l]);
        c->launches += 2;
        CK(cudaGetLastError());
        if (l > 0)
        {
            // gradient at this layer's input: the adjoint layer applied to g
            float2* dst = (gcur == n->gbuf[0]) ? n->gbuf[1] : n->gbuf[0];
            ST(lp_layer(c, l, true, nrhs, conf_d, gcur, lg, dst, lh));
            gcur = dst;
            lg = lh;
        }
    }
    if (loss_out)
    {
        CK(cudaMemcpyAsync(loss_out, n->dloss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return DWF_OK;
}

int lp_adam(dwf_ctx* c, double lr)
{
    LpNet* n = c->lp;
    n->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const double c1 = 1.0 / (1.0 - std::pow(double(b1), double(n->adam_t)));
    const double c2 = 1.0 / (1.0 - std::pow(double(b2), double(n->adam_t)));
    const long nr = 2 * n->woff[kLpLayers];
    lp_adam_kernel<<<grid_for(nr, c->nsm), 256, 0, c->stream>>>(
        reinterpret_cast<float*>(n->W), reinterpret_cast<const float*>(n->G), n->m, n->v, nr,
        float(lr), b1, b2, float(c1), float(c2), 1e-8f);
    c->launches += 1;
    CK(cudaGetLastError());
    return lp_pack(c);
}

int lp_ensure_solver(dwf_ctx* c, int nrhs)
{
    LpNet* n = c->lp;
    if (nrhs <= n->s_rhs)
        return DWF_OK;
    const size_t fs = size_t(nrhs) * c->fsz();
    for (int k = 0; k < 9; ++k)
        ST(lp_grow(c, n->s_f32[k], fs));
    ST(lp_grow(c, n->s_r64, fs));
    ST(lp_grow(c, n->s_t64, fs));
    ST(lp_grow(c, n->s_rhs64, fs));
    ST(lp_grow(c, n->s_part2, size_t(3) * nrhs * 64));
    ST(lp_grow(c, n->s_part, size_t(nrhs) * 64));
    ST(lp_grow(c, n->s_val, size_t(4) * nrhs));
    ST(lp_grow(c, n->s_state, size_t(nrhs)));
    n->s_rhs = nrhs;
    return DWF_OK;
}

// GCR workspace for nrhs right-hand sides and restart length m.
int lp_ensure_gcr(dwf_ctx* c, int nrhs, int m)
{
    LpNet* n = c->lp;
    const size_t need = size_t(m) * size_t(nrhs) * c->fsz();
    if (need > n->g_cap)
    {
        ST(lp_grow(c, n->g_Z, need));
        ST(lp_grow(c, n->g_W, need));
        n->g_cap = need;
    }
    if (nrhs > n->g_rhs)
    {
        ST(lp_grow(c, n->g_state, size_t(nrhs)));
        ST(lp_grow(c, n->g_flags, size_t(3) * nrhs));
        ST(lp_grow(c, n->g_part, size_t(nrhs) * 64 * 64));
        n->g_rhs = nrhs;
    }
    return DWF_OK;
}

// 256-thread launch as a programmatic dependent of the previous kernel on the
// stream (the kernel waits for it with griddepcontrol.wait before its first
// access); launch errors surface at the caller's cudaGetLastError.
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = grid;
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

template <int K>
void gcr_passes(const GcrArgs& g, dim3 grid, cudaStream_t s)
{
    launch_pdl(lp_gcr_dots_kernel<K>, grid, s, g);
    launch_pdl(lp_gcr_update_kernel<K>, grid, s, g);
}

void gcr_passes_k(int k, const GcrArgs& g, dim3 grid, cudaStream_t s)
{
    switch (k)
    {
#define DWFB_GCR_K(K)                    \
    case K:                              \
        gcr_passes<K>(g, grid, s);       \
        break;
        DWFB_GCR_K(0) DWFB_GCR_K(1) DWFB_GCR_K(2) DWFB_GCR_K(3) DWFB_GCR_K(4) DWFB_GCR_K(5)
        DWFB_GCR_K(6) DWFB_GCR_K(7) DWFB_GCR_K(8) DWFB_GCR_K(9) DWFB_GCR_K(10) DWFB_GCR_K(11)
        DWFB_GCR_K(12) DWFB_GCR_K(13) DWFB_GCR_K(14) DWFB_GCR_K(15)
#undef DWFB_GCR_K
    default:
        break;
    }
}

// Inner solve D e = r (FP32, r normalised by the caller) by flexible GCR(m)
// right-preconditioned by the network, for the right-hand sides with
// go[k] != 0, until |r|^2 <= tgt2 or inner_max iterations; e into x32, r
// overwritten by the final residual, iterations per right-hand side into its.
// Chunks of four iterations (with the end-of-cycle update of x32 in the last
// chunk of a cycle) are captured once into CUDA graphs and replayed; the
// first chunk of each inner solve runs directly (it also settles the Dslash
// autotuner).
int lp_gcr_inner(dwf_ctx* c, int nrhs, const int* conf_d, const std::vector<int>& go, double tgt2, float2* r,
                 float2* x32, std::vector<int>& its)
{
    LpNet* n = c->lp;
    const int m = n->gcr_m;
    const long fs = c->fsz();
    const long nf = fs * nrhs;
    ST(lp_ensure_gcr(c, nrhs, m));
    const int nblk = std::max(1, std::min(64, (4 * c->nsm + nrhs - 1) / nrhs));
    const bool chain = lp_chain(c, false);
    const int planes0 = cpad_of(n->C0) / 4;
    GcrArgs g;
    g.f4 = fs / 2;
    g.slot4 = nf / 2;
    g.nblk = nblk;
    g.W = reinterpret_cast<float4*>(n->g_W);
    g.Z = reinterpret_cast<const float4*>(n->g_Z);
    g.r = reinterpret_cast<float4*>(r);
    g.x = reinterpret_cast<float4*>(x32);
    g.planar = chain ? n->hb[0] : nullptr;
    g.Ls = c->L.Ls;
    g.V = c->L.V;
    g.planes = planes0;
    g.S = n->g_state;
    g.flags = n->g_flags;
    g.part = n->g_part;
    g.tgt2 = tgt2;
    g.maxit = n->inner_max;
    const dim3 grid(nblk, nrhs);

    // start: x32 = 0, |r|^2 and the active flags, the network's planar input
    CK(cudaMemsetAsync(x32, 0, size_t(nf) * sizeof(float2), c->stream));
    CK(cudaMemcpyAsync(n->g_flags + 2 * nrhs, go.data(), nrhs * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    const int dblk = int(std::min<long>(64, (fs + 4095) / 4096));
    lp_dots_kernel<<<dim3(dblk, nrhs), 256, 0, c->stream>>>(Dot{r, r}, Dot{r, r}, Dot{r, r}, 1, fs, dblk,
                                                            n->s_part2);
    lp_gcr_init_kernel<<<(nrhs + 127) / 128, 128, 0, c->stream>>>(n->s_part2, nrhs, dblk, n->g_state,
                                                                  n->g_flags + 2 * nrhs, n->g_flags, tgt2);
    c->launches += 2;
    if (chain)
    {
        lp_to_planar_kernel<<<grid_for(long(nrhs) * planes0 * c->L.V, c->nsm), 256, 0, c->stream>>>(
            r, op_layout(c), n->C0, planes0, c->L.V, nrhs, n->hb[0]);
        c->launches += 1;
    }
    CK(cudaGetLastError());

    auto iter = [&](int k) -> int {
        float2* zk = n->g_Z + size_t(k) * nf;
        float2* wk = n->g_W + size_t(k) * nf;
        if (chain)
            ST(lp_net(c, false, nrhs, conf_d, r, zk, false, true));
        else
            ST(lp_net(c, false, nrhs, conf_d, r, zk, false));
        ST(apply_dev(c, DWF_OP_D, nrhs, conf_d, 0, zk, wk, 32));
        gcr_passes_k(k, g, grid, c->stream);
        c->launches += 2;
        CK(cudaGetLastError());
        return DWF_OK;
    };
    auto chunk = [&](int k0) -> int {
        for (int k = k0; k < k0 + 4; ++k)
            ST(iter(k));
        if (k0 + 4 == m)
        {
            launch_pdl(lp_gcr_x_kernel, grid, c->stream, g, m);
            c->launches += 1;
        }
        CK(cudaGetLastError());
        return DWF_OK;
    };
    std::vector<int> fl(2 * nrhs, 0);
    int kc = 0;  // iterations of the current cycle already launched
    for (int done = 0; done < n->inner_max; done += 4)
    {
        const int k0 = kc;
        const int slot = k0 / 4;
        const std::vector<uintptr_t> key = {
            uintptr_t(nrhs), uintptr_t(chain), uintptr_t(m), uintptr_t(k0), uintptr_t(n->g_Z), uintptr_t(n->g_W),
            uintptr_t(n->g_state), uintptr_t(n->g_part), uintptr_t(r), uintptr_t(x32), uintptr_t(n->hb[0]),
            uintptr_t(n->act_rhs), uintptr_t(n->T), uintptr_t(conf_d), uintptr_t(c->U32),
            uintptr_t(lp_eff_variant(n) + 1), uintptr_t(std::llround(std::log10(tgt2) * 1000.0)),
            uintptr_t(n->inner_max), uintptr_t(nblk), uintptr_t(c->dslash_variant)};
        if (done == 0)
            ST(chunk(k0));
        else if (n->gcr_exec[slot] && n->gcr_key[slot] == key)
        {
            CK(cudaGraphLaunch(n->gcr_exec[slot], c->stream));
            c->launches += n->gcr_nodes[slot];
        }
        else
        {
            if (n->gcr_exec[slot])
            {
                cudaGraphExecDestroy(n->gcr_exec[slot]);
                n->gcr_exec[slot] = nullptr;
            }
            const uint64_t l0 = c->launches;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            const int st = chunk(k0);
            cudaGraph_t gr = nullptr;
            const cudaError_t e = cudaStreamEndCapture(c->stream, &gr);
            if (st != DWF_OK || e != cudaSuccess)
            {
                if (gr)
                    cudaGraphDestroy(gr);
                return st != DWF_OK ? st : ctx_fail(c, DWF_CUDA_ERROR, "learned: GCR graph capture failed");
            }
            const cudaError_t e2 = cudaGraphInstantiate(&n->gcr_exec[slot], gr, 0);
            cudaGraphDestroy(gr);
            if (e2 != cudaSuccess)
            {
                n->gcr_exec[slot] = nullptr;
                return ctx_fail(c, DWF_CUDA_ERROR, "learned: GCR graph instantiation failed");
            }
            n->gcr_key[slot] = key;
            n->gcr_nodes[slot] = c->launches - l0;
            CK(cudaGraphLaunch(n->gcr_exec[slot], c->stream));
        }
        kc = (k0 + 4 == m) ? 0 : k0 + 4;
        CK(cudaMemcpyAsync(fl.data(), n->g_flags, 2 * nrhs * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        bool any = false;
        for (int k = 0; k < nrhs; ++k)
            any = any || fl[k];
        if (!any)
            break;
    }
    if (kc != 0)
    {
        // a cycle cut short: its correction from the iterations launched
        launch_pdl(lp_gcr_x_kernel, grid, c->stream, g, kc);
        c->launches += 1;
        CK(cudaMemcpyAsync(fl.data(), n->g_flags, 2 * nrhs * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    CK(cudaGetLastError());
    its.assign(fl.begin() + nrhs, fl.begin() + 2 * nrhs);
    return DWF_OK;
}

// DWF_TIMEOUT (and the flag cleared) if a tcgen05 layer gave up a bounded wait.
int lp_check_err(dwf_ctx* c)
{
    int e = 0;
    CK(cudaMemcpyAsync(&e, c->lp->err_d, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (e)
    {
        CK(cudaMemsetAsync(c->lp->err_d, 0, sizeof(int), c->stream));
        return ctx_fail(c, DWF_TIMEOUT, "learned: a tensor-core layer timed out waiting for its MMAs");
    }
    return DWF_OK;
}

// Gaussian FP64 fields (n complex numbers) on the device.
int lp_gauss(dwf_ctx* c, double2* out, long n, uint64_t seed)
{
    lp_gauss_kernel<<<grid_for(n, c->nsm), 256, 0, c->stream>>>(out, n, seed);
    c->launches += 1;
    CK(cudaGetLastError());
    return DWF_OK;
}

}  // namespace

void lp_destroy(dwf_ctx* c)
{
    LpNet* n = c->lp;
    if (!n)
        return;
    void* bufs[] = {n->W, n->G, n->m, n->v, n->Bf, n->Ba, n->Btf, n->Bta, n->err_d, n->hb[0], n->hb[1], n->T, n->act[1], n->act[2], n->act[3],
                    n->hid[0], n->hid[1], n->gbuf[0], n->gbuf[1], n->gpart, n->lpart, n->lscale,
                    n->dloss, n->dconf, n->pr_rho, n->pr_e, n->s_r64, n->s_t64, n->s_rhs64,
                    n->s_part2, n->s_part, n->s_val, n->s_state};
    for (void* b : bufs)
        if (b)
            cudaFree(b);
    for (float2* b : n->s_f32)
        if (b)
            cudaFree(b);
    void* gbufs[] = {n->g_Z, n->g_W, n->g_state, n->g_flags, n->g_part};
    for (void* b : gbufs)
        if (b)
            cudaFree(b);
    if (n->g_exec)
        cudaGraphExecDestroy(n->g_exec);
    for (cudaGraphExec_t ge : n->gcr_exec)
        if (ge)
            cudaGraphExecDestroy(ge);
    delete n;
    c->lp = nullptr;
}

// Solve D x = src for nrhs sources: FP64 defect correction around an FP32
// inner solve right-preconditioned by the network (flexible GCR(m), or
// BiCGStab), then (for right-hand sides that stall) the mixed CG on D^dag D
// from the current iterate.
// Automatic layer kernel (variant -1): the first solve per batch-size bucket
// times one network application with each kernel (CUDA events, after a
// warm-up) and keeps the faster; the tcgen05 kernel competes only where every
// layer's tile fits. Uses the solver's scratch fields.
int lp_tune_variant(dwf_ctx* c, int nrhs, const int* conf_d)
{
    LpNet* n = c->lp;
    int bucket = 0;
    while ((1 << bucket) < nrhs && bucket < 20)
        ++bucket;
    const auto it = n->auto_tuned.find(bucket);
    if (it != n->auto_tuned.end())
    {
        n->auto_variant = it->second;
        return DWF_OK;
    }
    bool tc_all = true;
    for (int l = 0; l < kLpLayers; ++l)
        tc_all = tc_all && tc_fits(c, l, false) && tc_fits(c, l, true);
    int choice = 0;
    if (tc_all)
    {
        const long nf = long(nrhs) * c->fsz();
        ST(lp_gauss(c, n->s_r64, nf, 777));
        lp_f64_to_f32_kernel<<<grid_for(nf, c->nsm), 256, 0, c->stream>>>(n->s_r64, n->s_f32[0], nf);
        c->launches += 1;
        float best = 1e30f;
        for (int v = 0; v <= 1; ++v)
        {
            n->auto_variant = v;
            ST(lp_net(c, false, nrhs, conf_d, n->s_f32[0], n->s_f32[1], false));  // warm-up
            CK(cudaEventRecord(c->ev0, c->stream));
            for (int r = 0; r < 3; ++r)
                ST(lp_net(c, false, nrhs, conf_d, n->s_f32[0], n->s_f32[1], false));
            CK(cudaEventRecord(c->ev1, c->stream));
            CK(cudaEventSynchronize(c->ev1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
            if (ms < best)
            {
                best = ms;
                choice = v;
            }
        }
        ST(lp_check_err(c));
    }
    n->auto_tuned[bucket] = choice;
    n->auto_variant = choice;
    return DWF_OK;
}

int lp_solve(dwf_ctx* c, int nrhs, const int* conf_h, const double2* src, double2* x,
             double rtol, int maxiter, dwf_solve_info* info)
{
    LpNet* n = c->lp;
    if (!n)
        return ctx_fail(c, DWF_BAD_ARG, "learned solver: no network (dwf_lp_init first)");
    if (nrhs < 1 || nrhs > 65535)
        return ctx_fail(c, DWF_BAD_ARG, "learned solver: nrhs out of range");
    const int* conf_d = nullptr;
    ST(lp_conf(c, nrhs, conf_h, &conf_d));
    ST(lp_transports(c));
    ST(lp_ensure_solver(c, nrhs));
    // the fused update kernels write the network's planar input (hb[0]) before
    // the network runs: size the activation buffers for this batch first
    ST(lp_ensure_act(c, nrhs));
    if (n->variant < 0)
        ST(lp_tune_variant(c, nrhs, conf_d));
    const long fs = c->fsz();
    const long nf = fs * nrhs;
    const int nblk = int(std::min<long>(64, (fs + 4095) / 4096));
    float2 *r = n->s_f32[0], *rh = n->s_f32[1], *p = n->s_f32[2], *v = n->s_f32[3], *s = n->s_f32[4],
           *t = n->s_f32[5], *ph = n->s_f32[6], *sh = n->s_f32[7], *x32 = n->s_f32[8];
    double* val = n->s_val;  // [0] |r64|^2, [1] |D^dag r64|^2, [2] inverse norms, [3] scales
    const dim3 rgrid(nblk, nrhs);
    const int vgrid = grid_for(nf, c->nsm);
    const int sgrid = (nrhs + 127) / 128;

    // |D^dag src|^2 (stopping-rule denominator)
    ST(apply_dev(c, DWF_OP_DDAG, nrhs, conf_d, 0, src, n->s_t64, 64));
    lp_norm_kernel<<<rgrid, 256, 0, c->stream>>>(n->s_t64, fs, nblk, n->s_part);
    lp_sum_kernel<<<sgrid, 128, 0, c->stream>>>(n->s_part, nrhs, nblk, val + 1);
    c->launches += 2;
    std::vector<double> bnorm2(nrhs), rnorm2(nrhs), nrm2(nrhs), prev(nrhs, -1.0), scale(nrhs);
    CK(cudaMemcpyAsync(bnorm2.data(), val + 1, nrhs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemsetAsync(x, 0, size_t(nf) * sizeof(double2), c->stream));
    CK(cudaStreamSynchronize(c->stream));

    std::vector<int> done(nrhs, 0), stalled(nrhs, 0), iters(nrhs, 0), cycles(nrhs, 0);
    std::vector<BsState> hs(nrhs);
    std::vector<double> relres(nrhs, 1.0);
    const double tgt2 = n->inner_tol * n->inner_tol;
    long total_inner = 0;
    for (int cyc = 0; cyc <= n->outer_max; ++cyc)
    {
        // r64 = src - D x; measure |D^dag r64| / |D^dag src|
        ST(apply_dev(c, DWF_OP_D, nrhs, conf_d, 0, x, n->s_t64, 64));
        lp_resid_kernel<<<rgrid, 256, 0, c->stream>>>(src, n->s_t64, n->s_r64, fs, nblk, n->s_part);
        lp_sum_kernel<<<sgrid, 128, 0, c->stream>>>(n->s_part, nrhs, nblk, val);
        ST(apply_dev(c, DWF_OP_DDAG, nrhs, conf_d, 0, n->s_r64, n->s_t64, 64));
        lp_norm_kernel<<<rgrid, 256, 0, c->stream>>>(n->s_t64, fs, nblk, n->s_part);
        lp_sum_kernel<<<sgrid, 128, 0, c->stream>>>(n->s_part, nrhs, nblk, val + nrhs);
        c->launches += 4;
        CK(cudaMemcpyAsync(rnorm2.data(), val, nrhs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(nrm2.data(), val + nrhs, nrhs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        int left = 0;
        for (int k = 0; k < nrhs; ++k)
        {
            relres[k] = bnorm2[k] > 0.0 ? std::sqrt(nrm2[k] / bnorm2[k]) : 0.0;
            if (!std::isfinite(relres[k]))
                stalled[k] = 1;
            if (relres[k] <= rtol)
                done[k] = 1;
            // stall: the true residual fell by less than a factor 2 in a cycle
            if (!done[k] && prev[k] >= 0.0 && relres[k] > 0.5 * prev[k])
                stalled[k] = 1;
            if (!done[k] && iters[k] >= maxiter)
                stalled[k] = 1;
            prev[k] = relres[k];
            const bool go = !done[k] && !stalled[k];
            left += go ? 1 : 0;
            const double rn = std::sqrt(rnorm2[k]);
            scale[k] = go && rn > 0.0 ? rn : 0.0;
            hs[k].active = go ? 1 : 0;
        }
        if (!left || cyc == n->outer_max)
            break;
        // inner system D e = r64 / |r64| in FP32
        std::vector<double> inv(nrhs);
        for (int k = 0; k < nrhs; ++k)
            inv[k] = scale[k] > 0.0 ? 1.0 / scale[k] : 0.0;
        CK(cudaMemcpyAsync(val + 2 * nrhs, inv.data(), nrhs * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(val + 3 * nrhs, scale.data(), nrhs * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        lp_down_kernel<<<vgrid, 256, 0, c->stream>>>(n->s_r64, val + 2 * nrhs, fs, nrhs, r);
        c->launches += 1;
        std::vector<int> inner_its(nrhs, 0);
        if (n->krylov == 0)
        {
            std::vector<int> go(nrhs);
            for (int k = 0; k < nrhs; ++k)
                go[k] = hs[k].active;
            ST(lp_gcr_inner(c, nrhs, conf_d, go, tgt2, r, x32, inner_its));
        }
        else
        {
            CK(cudaMemcpyAsync(n->s_state, hs.data(), nrhs * sizeof(BsState), cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemcpyAsync(rh, r, size_t(nf) * sizeof(float2), cudaMemcpyDeviceToDevice, c->stream));
            CK(cudaMemsetAsync(p, 0, size_t(nf) * sizeof(float2), c->stream));
            CK(cudaMemsetAsync(v, 0, size_t(nf) * sizeof(float2), c->stream));
            CK(cudaMemsetAsync(x32, 0, size_t(nf) * sizeof(float2), c->stream));
            lp_dots_kernel<<<rgrid, 256, 0, c->stream>>>(Dot{rh, r}, Dot{r, r}, Dot{r, r}, 2, fs, nblk, n->s_part2);
            lp_bs_coef_kernel<<<sgrid, 128, 0, c->stream>>>(0, n->s_part2, nrhs, nblk, n->s_state, tgt2, n->inner_max);
            c->launches += 2;
            // one BiCGStab iteration; the coefficient kernels read the dot products
            // of the previous kernel (slots 0, 1 of s_part2)
            const bool chain = lp_chain(c, false);
            const int planes0 = cpad_of(n->C0) / 4;
            const int pgrid = grid_for(long(nrhs) * planes0 * c->L.V, c->nsm);
            auto body = [&]() -> int {
                lp_bs_coef_kernel<<<sgrid, 128, 0, c->stream>>>(1, n->s_part2, nrhs, nblk, n->s_state, tgt2, n->inner_max);
                if (chain)
                {
                    lp_bs_planar_kernel<<<pgrid, 256, 0, c->stream>>>(0, c->L.Ls, c->L.V, planes0, nrhs, n->s_state, p, r,
                                                                      v, s, n->hb[0]);
                    ST(lp_net(c, false, nrhs, conf_d, p, ph, false, true));
                }
                else
                {
                    lp_bs_vec_kernel<<<vgrid, 256, 0, c->stream>>>(0, fs, nrhs, n->s_state, p, r, v, s, x32, ph, sh, t, r);
                    ST(lp_net(c, false, nrhs, conf_d, p, ph, false));
                }
                ST(apply_dev(c, DWF_OP_D, nrhs, conf_d, 0, ph, v, 32));
                lp_dots_kernel<<<rgrid, 256, 0, c->stream>>>(Dot{rh, v}, Dot{rh, v}, Dot{rh, v}, 1, fs, nblk, n->s_part2);
                lp_bs_coef_kernel<<<sgrid, 128, 0, c->stream>>>(2, n->s_part2, nrhs, nblk, n->s_state, tgt2, n->inner_max);
                if (chain)
                {
                    lp_bs_planar_kernel<<<pgrid, 256, 0, c->stream>>>(1, c->L.Ls, c->L.V, planes0, nrhs, n->s_state, p, r,
                                                                      v, s, n->hb[0]);
                    ST(lp_net(c, false, nrhs, conf_d, s, sh, false, true));
                }
                else
                {
                    lp_bs_vec_kernel<<<vgrid, 256, 0, c->stream>>>(1, fs, nrhs, n->s_state, p, r, v, s, x32, ph, sh, t, r);
                    ST(lp_net(c, false, nrhs, conf_d, s, sh, false));
                }
                ST(apply_dev(c, DWF_OP_D, nrhs, conf_d, 0, sh, t, 32));
                lp_dots_kernel<<<rgrid, 256, 0, c->stream>>>(Dot{t, s}, Dot{t, t}, Dot{t, t}, 2, fs, nblk, n->s_part2);
                lp_bs_coef_kernel<<<sgrid, 128, 0, c->stream>>>(3, n->s_part2, nrhs, nblk, n->s_state, tgt2, n->inner_max);
                lp_bs_xr_kernel<<<rgrid, 256, 0, c->stream>>>(fs, nblk, n->s_state, x32, ph, sh, s, t, r, rh, n->s_part2);
                c->launches += 8;
                CK(cudaGetLastError());
                return DWF_OK;
            };
            const int chunk = 4;
            // the chunk of iterations is captured once into a CUDA graph and replayed;
            // the first chunk runs directly (it also settles the Dslash autotuner)
            const std::vector<uintptr_t> key = {uintptr_t(nrhs), uintptr_t(chain), uintptr_t(n->s_rhs),
                                                uintptr_t(n->act_rhs), uintptr_t(n->T), uintptr_t(conf_d),
                                                uintptr_t(c->U32), uintptr_t(lp_eff_variant(n) + 1),
                                                uintptr_t(std::llround(std::log10(tgt2) * 1000.0)),
                                                uintptr_t(n->inner_max), uintptr_t(nblk), uintptr_t(c->dslash_variant)};
            for (int it = 0; it < n->inner_max; it += chunk)
            {
                if (it > 0 && n->g_exec && n->g_key == key)
                {
                    CK(cudaGraphLaunch(n->g_exec, c->stream));
                    c->launches += n->g_nodes;
                }
                else if (it > 0)
                {
                    if (n->g_exec)
                    {
                        cudaGraphExecDestroy(n->g_exec);
                        n->g_exec = nullptr;
                    }
                    const uint64_t l0 = c->launches;
                    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                    int st = DWF_OK;
                    for (int u = 0; u < chunk && st == DWF_OK; ++u)
                        st = body();
                    cudaGraph_t g = nullptr;
                    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
                    if (st != DWF_OK || e != cudaSuccess)
                    {
                        if (g)
                            cudaGraphDestroy(g);
                        return st != DWF_OK ? st : ctx_fail(c, DWF_CUDA_ERROR, "learned: graph capture failed");
                    }
                    const cudaError_t e2 = cudaGraphInstantiate(&n->g_exec, g, 0);
                    cudaGraphDestroy(g);
                    if (e2 != cudaSuccess)
                    {
                        n->g_exec = nullptr;
                        return ctx_fail(c, DWF_CUDA_ERROR, "learned: graph instantiation failed");
                    }
                    n->g_key = key;
                    n->g_nodes = c->launches - l0;
                    CK(cudaGraphLaunch(n->g_exec, c->stream));
                }
                else
                {
                    for (int u = 0; u < chunk; ++u)
                        ST(body());
                }
                CK(cudaMemcpyAsync(hs.data(), n->s_state, nrhs * sizeof(BsState), cudaMemcpyDeviceToHost, c->stream));
                CK(cudaStreamSynchronize(c->stream));
                bool any = false;
                for (int k = 0; k < nrhs; ++k)
                    any = any || hs[k].active;
                if (!any)
                    break;
            }
            // the last coefficient step leaves rr of the final r; stop flags too
            lp_dots_kernel<<<rgrid, 256, 0, c->stream>>>(Dot{rh, r}, Dot{r, r}, Dot{r, r}, 2, fs, nblk, n->s_part2);
            c->launches += 1;
            CK(cudaMemcpyAsync(hs.data(), n->s_state, nrhs * sizeof(BsState), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            for (int k = 0; k < nrhs; ++k)
                inner_its[k] = hs[k].iters;
        }
        lp_up_kernel<<<vgrid, 256, 0, c->stream>>>(x, x32, val + 3 * nrhs, fs, nrhs);
        c->launches += 1;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(c->stream));
        ST(lp_check_err(c));
        for (int k = 0; k < nrhs; ++k)
            if (scale[k] > 0.0)
            {
                iters[k] += inner_its[k];
                cycles[k] += 1;
                total_inner += inner_its[k];
            }
    }
    n->iters_total += total_inner;
    // fallback: mixed CG on D^dag D from the current iterate
    std::vector<int> fb(nrhs, 0);
    int nfb = 0;
    for (int k = 0; k < nrhs; ++k)
        if (!done[k])
        {
            fb[k] = 1;
            ++nfb;
        }
    std::vector<dwf_solve_info> fbi(nrhs);
    if (nfb)
    {
        ST(apply_dev(c, DWF_OP_DDAG, nrhs, conf_d, 0, src, n->s_rhs64, 64));
        ST(solve_batch(c, DWF_OP_DDAGD, nrhs, conf_h, n->s_rhs64, x, 1, rtol, maxiter,
                       DWF_SOLVER_MIXED, 0, fbi.data()));
    }
    else
    {
        // every right-hand side met the rule on the FP64 true residual above
        for (int k = 0; k < nrhs; ++k)
            fbi[k].true_relres = relres[k];
    }
    for (int k = 0; info && k < nrhs; ++k)
    {
        dwf_solve_info& I = info[k];
        I.iterations = iters[k] + (fb[k] ? fbi[k].iterations : 0);
        I.true_relres = fbi[k].true_relres;
        I.relres = fb[k] ? fbi[k].relres : relres[k];
        I.status = fb[k] ? fbi[k].status : DWF_OK;
        if (I.status == DWF_OK && !(I.true_relres <= rtol))
            I.status = std::isfinite(I.true_relres) ? DWF_NOT_CONVERGED : DWF_NONFINITE;
        I.converged = I.status == DWF_OK ? 1 : 0;
        I.solver = DWF_SOLVER_LEARNED;
        I.reliable_updates = cycles[k];
        I.fallback = fb[k];
        I.dirac_relres = 0.0;
        I.schur_iterations = iters[k];  // preconditioned iterations (GCR: 1 network + 1 D each; BiCGStab: 2 + 2)
    }
    return DWF_OK;
}

}  // namespace dwfb

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int dwf_lp_init(dwf_ctx* c, int hidden, uint64_t seed)
{
    if (!c)
        return DWF_BAD_ARG;
    if (hidden != 8 && hidden != 16 && hidden != 24 && hidden != 32)
        return ctx_fail(c, DWF_BAD_ARG, "dwf_lp_init: hidden must be 8, 16, 24 or 32");
    const int C0 = 2 * c->L.Ls;
    if (C0 > 48 || C0 * hidden > kGradThreads * kGradMaxPer)
        return ctx_fail(c, DWF_BAD_ARG, "dwf_lp_init: 2*Ls*hidden must be <= 1536 and Ls <= 24");
    CK(cudaSetDevice(c->device));
    lp_destroy(c);
    LpNet* n = new LpNet();
    c->lp = n;
    n->C0 = C0;
    n->H = hidden;
    const int ch[kLpLayers + 1] = {C0, hidden, hidden, hidden, C0};
    n->woff[0] = n->bf_off[0] = n->ba_off[0] = 0;
    for (int l = 0; l < kLpLayers; ++l)
    {
        n->cin[l] = ch[l];
        n->cout[l] = ch[l + 1];
        n->ntf[l] = nt_of(ch[l + 1]);
        n->nta[l] = nt_of(ch[l]);
        n->woff[l + 1] = n->woff[l] + 9L * ch[l] * ch[l + 1];
        n->bf_off[l + 1] = n->bf_off[l] + 9L * (cpad_of(ch[l]) / 8) * n->ntf[l] * 32;
        n->ba_off[l + 1] = n->ba_off[l] + 9L * (cpad_of(ch[l + 1]) / 8) * n->nta[l] * 32;
        n->ncf[l] = ncol_of(ch[l + 1]);
        n->nca[l] = ncol_of(ch[l]);
        if (l == 0)
            n->tf_off[0] = n->ta_off[0] = 0;
        n->tf_off[l + 1] = n->tf_off[l] + 9L * (cpad_of(ch[l]) / 8) * 2 * n->ncf[l];
        n->ta_off[l + 1] = n->ta_off[l] + 9L * (cpad_of(ch[l + 1]) / 8) * 2 * n->nca[l];
    }
    const long nw = n->woff[kLpLayers];
    ST(lp_grow(c, n->W, nw));
    ST(lp_grow(c, n->G, nw));
    ST(lp_grow(c, n->m, 2 * nw));
    ST(lp_grow(c, n->v, 2 * nw));
    ST(lp_grow(c, n->Bf, n->bf_off[kLpLayers]));
    ST(lp_grow(c, n->Ba, n->ba_off[kLpLayers]));
    ST(lp_grow(c, n->Btf, n->tf_off[kLpLayers]));
    ST(lp_grow(c, n->Bta, n->ta_off[kLpLayers]));
    ST(lp_grow(c, n->err_d, 1));
    CK(cudaMemsetAsync(n->err_d, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(n->m, 0, 2 * nw * sizeof(float), c->stream));
    CK(cudaMemsetAsync(n->v, 0, 2 * nw * sizeof(float), c->stream));
    // initial weights: small seeded Gaussian noise, plus the identity on the
    // centre offset of each layer (scaled 1/2 in the first), so that N starts
    // close to a multiple of the identity on the channels every layer keeps
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<float2> w(nw);
    for (int l = 0; l < kLpLayers; ++l)
    {
        const double sd = 0.02 / std::sqrt(9.0 * n->cin[l]);
        for (long i = n->woff[l]; i < n->woff[l + 1]; ++i)
        {
            const double re = nd(gen) * sd;
            const double im = nd(gen) * sd;
            w[i] = make_float2(float(re), float(im));
        }
        for (int o = 0; o < std::min(n->cin[l], n->cout[l]); ++o)
            w[n->woff[l] + long(o) * n->cin[l] + o].x += (l == 0) ? 0.5f : 1.0f;
    }
    CK(cudaMemcpyAsync(n->W, w.data(), nw * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    ST(lp_pack(c));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int dwf_lp_weights_size(const dwf_ctx* c, long* n_complex)
{
    if (!c || !c->lp || !n_complex)
        return DWF_BAD_ARG;
    *n_complex = c->lp->woff[kLpLayers];
    return DWF_OK;
}

int dwf_lp_get_weights(dwf_ctx* c, float* w)
{
    if (!c || !c->lp || !w)
        return DWF_BAD_ARG;
    CK(cudaMemcpyAsync(w, c->lp->W, c->lp->woff[kLpLayers] * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int dwf_lp_set_weights(dwf_ctx* c, const float* w)
{
    if (!c || !c->lp || !w)
        return DWF_BAD_ARG;
    CK(cudaMemcpyAsync(c->lp->W, w, c->lp->woff[kLpLayers] * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    c->lp->adam_t = 0;
    CK(cudaMemsetAsync(c->lp->m, 0, 2 * c->lp->woff[kLpLayers] * sizeof(float), c->stream));
    CK(cudaMemsetAsync(c->lp->v, 0, 2 * c->lp->woff[kLpLayers] * sizeof(float), c->stream));
    ST(lp_pack(c));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int dwf_lp_transports(dwf_ctx* c, int conf, float* T)
{
    if (!c || !c->lp || !T || conf < 0 || conf >= c->nconf)
        return DWF_BAD_ARG;
    ST(lp_transports(c));
    CK(cudaMemcpyAsync(T, c->lp->T + long(conf) * c->L.V * 9, size_t(c->L.V) * 9 * sizeof(float2),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DWF_OK;
}

int dwf_lp_apply_dev(dwf_ctx* c, int adjoint, int nrhs, const int* rhs_conf, const void* in, void* out)
{
    if (!c || !c->lp || !in || !out || nrhs < 1 || nrhs > 65535)
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_apply_dev: bad arguments or no network") : DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    const int* conf_d = nullptr;
    ST(lp_conf(c, nrhs, rhs_conf, &conf_d));
    ST(lp_transports(c));
    ST(lp_net(c, adjoint != 0, nrhs, conf_d, static_cast<const float2*>(in), static_cast<float2*>(out), false));
    return lp_check_err(c);
}

int dwf_lp_layer_dev(dwf_ctx* c, int layer, int adjoint, int nrhs, const int* rhs_conf, const void* in,
                     void* out)
{
    if (!c || !c->lp || !in || !out || nrhs < 1 || nrhs > 65535 || layer < 0 || layer >= kLpLayers)
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_layer_dev: bad arguments or no network") : DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    const int* conf_d = nullptr;
    ST(lp_conf(c, nrhs, rhs_conf, &conf_d));
    ST(lp_transports(c));
    LpNet* n = c->lp;
    const int ci = adjoint ? n->cout[layer] : n->cin[layer];
    const int co = adjoint ? n->cin[layer] : n->cout[layer];
    ST(lp_layer(c, layer, adjoint != 0, nrhs, conf_d, static_cast<const float2*>(in), net_layout(c, ci),
                static_cast<float2*>(out), net_layout(c, co)));
    return lp_check_err(c);
}

int dwf_lp_loss_grad_dev(dwf_ctx* c, int npair, const int* pair_conf, const void* rho, const void* e,
                         double* loss, float* grad)
{
    if (!c || !c->lp || !rho || !e || npair < 1 || npair > 1024)
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_loss_grad_dev: bad arguments or no network") : DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    const int* conf_d = nullptr;
    ST(lp_conf(c, npair, pair_conf, &conf_d));
    ST(lp_transports(c));
    ST(lp_loss_grad(c, npair, conf_d, static_cast<const float2*>(rho), static_cast<const float2*>(e), loss));
    ST(lp_check_err(c));
    if (grad)
    {
        CK(cudaMemcpyAsync(grad, c->lp->G, c->lp->woff[kLpLayers] * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return DWF_OK;
}

// Training pairs: for each configuration, `pairs_per_conf` pairs. A fraction
// come from the plain solver (error of a truncated CG iterate against the
// converged solution, rho = D e); the rest are e ~ Gaussian, rho = D e.
int dwf_lp_train(dwf_ctx* c, const dwf_lp_train_params* tp, dwf_lp_train_info* ti, double* history)
{
    if (!c || !c->lp || !tp || tp->steps < 0 || tp->batch < 1 || tp->batch > 1024 ||
        tp->pairs_per_conf < 1 || !(tp->lr > 0.0))
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_train: bad parameters or no network") : DWF_BAD_ARG;
    if (c->nconf < 1)
        return ctx_fail(c, DWF_BAD_ARG, "dwf_lp_train: no gauge configuration (set_gauge first)");
    CK(cudaSetDevice(c->device));
    LpNet* n = c->lp;
    const auto t0 = std::chrono::steady_clock::now();
    ST(lp_transports(c));
    const long fs = c->fsz();
    const int np = c->nconf * tp->pairs_per_conf;
    if (np != n->npairs)
    {
        ST(lp_grow(c, n->pr_rho, size_t(np) * fs));
        ST(lp_grow(c, n->pr_e, size_t(np) * fs));
        n->npairs = np;
    }
    n->pr_conf.assign(np, 0);
    for (int k = 0; k < np; ++k)
        n->pr_conf[k] = k / tp->pairs_per_conf;
    // generate pairs in groups of up to 16 (FP64 staging in the solver
    // workspace); group g is a solver group when g % solver_every == 0
    const int grp = std::min(np, 16);
    ST(lp_ensure_solver(c, grp));
    int nsolver = 0;
    const int* conf_d = nullptr;
    for (int k0 = 0; k0 < np; k0 += grp)
    {
        const int m = std::min(grp, np - k0);
        ST(lp_conf(c, m, n->pr_conf.data() + k0, &conf_d));
        const bool solver_pair = tp->solver_iters > 0 &&
                                 (k0 / grp) % std::max(1, tp->solver_every) == 0;
        ST(lp_gauss(c, n->s_r64, long(m) * fs, tp->seed * 0x100000001B3ull + uint64_t(k0)));
        if (solver_pair)
        {
            // b Gaussian; x* = converged CG solution of D^dag D x = D^dag b;
            // x_k = CG truncated at solver_iters; e = x* - x_k
            std::vector<int> cf(n->pr_conf.begin() + k0, n->pr_conf.begin() + k0 + m);
            ST(apply_dev(c, DWF_OP_DDAG, m, conf_d, 0, n->s_r64, n->s_rhs64, 64));
            std::vector<dwf_solve_info> inf(m);
            ST(solve_batch(c, DWF_OP_DDAGD, m, cf.data(), n->s_rhs64, n->s_t64, 0, 1e-8,
                           std::max(tp->solver_maxiter, 1), DWF_SOLVER_MIXED, 0, inf.data()));
            ST(solve_batch(c, DWF_OP_DDAGD, m, cf.data(), n->s_rhs64, n->s_r64, 0, 1e-30,
                           tp->solver_iters, DWF_SOLVER_CG64, 0, inf.data()));
            lp_diff_kernel<<<grid_for(long(m) * fs, c->nsm), 256, 0, c->stream>>>(
                n->s_t64, n->s_r64, n->pr_e + long(k0) * fs, long(m) * fs);
            nsolver += m;
        }
        else
            lp_f64_to_f32_kernel<<<grid_for(long(m) * fs, c->nsm), 256, 0, c->stream>>>(
                n->s_r64, n->pr_e + long(k0) * fs, long(m) * fs);
        c->launches += 1;
        CK(cudaGetLastError());
        ST(apply_dev(c, DWF_OP_D, m, conf_d, 0, n->pr_e + long(k0) * fs, n->pr_rho + long(k0) * fs, 32));
    }
    CK(cudaStreamSynchronize(c->stream));
    const auto t1 = std::chrono::steady_clock::now();
    // Adam over mini-batches drawn in a seeded shuffled order
    std::mt19937_64 gen(tp->seed ^ 0x5DEECE66Dull);
    std::vector<int> order(np);
    for (int k = 0; k < np; ++k)
        order[k] = k;
    const int B = std::min(tp->batch, np);
    ST(lp_ensure_act(c, B));
    float2* brho = nullptr;
    float2* be = nullptr;
    if (cudaMalloc(&brho, size_t(B) * fs * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&be, size_t(B) * fs * sizeof(float2)) != cudaSuccess)
    {
        cudaFree(brho);  // cudaFree(nullptr) is a no-op
        return ctx_fail(c, DWF_CUDA_ERROR, "dwf_lp_train: mini-batch allocation failed");
    }
    double first = -1.0, last = -1.0;
    int pos = np;
    std::vector<int> bc(B);
    int st = DWF_OK;
    for (int step = 0; step < tp->steps && st == DWF_OK; ++step)
    {
        if (pos + B > np)
        {
            std::shuffle(order.begin(), order.end(), gen);
            pos = 0;
        }
        for (int b = 0; b < B; ++b)
        {
            const int k = order[pos + b];
            bc[b] = n->pr_conf[k];
            cudaMemcpyAsync(brho + long(b) * fs, n->pr_rho + long(k) * fs, fs * sizeof(float2),
                            cudaMemcpyDeviceToDevice, c->stream);
            cudaMemcpyAsync(be + long(b) * fs, n->pr_e + long(k) * fs, fs * sizeof(float2),
                            cudaMemcpyDeviceToDevice, c->stream);
        }
        pos += B;
        st = lp_conf(c, B, bc.data(), &conf_d);
        const bool logit = history || step == 0 || step == tp->steps - 1;
        double L = 0.0;
        if (st == DWF_OK)
            st = lp_loss_grad(c, B, conf_d, brho, be, logit ? &L : nullptr);
        if (st == DWF_OK)
        {
            const double lr = tp->lr * (tp->lr_decay_steps > 0 ? std::pow(0.5, double(step) / tp->lr_decay_steps) : 1.0);
            st = lp_adam(c, lr);
        }
        if (logit)
        {
            if (first < 0.0)
                first = L;
            last = L;
            if (history)
                history[step] = L;
        }
    }
    cudaStreamSynchronize(c->stream);
    cudaFree(brho);
    cudaFree(be);
    if (st != DWF_OK)
        return st;
    ST(lp_check_err(c));
    const auto t2 = std::chrono::steady_clock::now();
    if (ti)
    {
        ti->loss_first = first;
        ti->loss_last = last;
        ti->steps = tp->steps;
        ti->npairs = np;
        ti->solver_pairs = nsolver;
        ti->seconds_pairs = std::chrono::duration<double>(t1 - t0).count();
        ti->seconds_train = std::chrono::duration<double>(t2 - t1).count();
    }
    return DWF_OK;
}

int dwf_lp_time_network(dwf_ctx* c, int nrhs, int reps, double* ms_per_apply, double* flops_per_apply)
{
    if (!c || !c->lp || nrhs < 1 || nrhs > 65535 || reps < 1 || !ms_per_apply)
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_time_network: bad arguments or no network") : DWF_BAD_ARG;
    if (c->nconf < 1)
        return ctx_fail(c, DWF_BAD_ARG, "dwf_lp_time_network: no gauge configuration");
    CK(cudaSetDevice(c->device));
    LpNet* n = c->lp;
    const int* conf_d = nullptr;
    ST(lp_conf(c, nrhs, nullptr, &conf_d));
    ST(lp_transports(c));
    ST(lp_ensure_solver(c, nrhs));
    ST(lp_ensure_act(c, nrhs));
    const long nf = long(nrhs) * c->fsz();
    ST(lp_gauss(c, n->s_r64, nf, 12345));
    lp_f64_to_f32_kernel<<<grid_for(nf, c->nsm), 256, 0, c->stream>>>(n->s_r64, n->s_f32[0], nf);
    c->launches += 1;
    ST(lp_net(c, false, nrhs, conf_d, n->s_f32[0], n->s_f32[1], false));  // warm-up
    CK(cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < reps; ++r)
        ST(lp_net(c, false, nrhs, conf_d, n->s_f32[0], n->s_f32[1], false));
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *ms_per_apply = double(ms) / reps;
    if (flops_per_apply)
    {
        double cc = 0.0;
        for (int l = 0; l < kLpLayers; ++l)
            cc += double(n->cin[l]) * n->cout[l];
        // 9 offsets, complex multiply-add = 8 real flops
        *flops_per_apply = 8.0 * 9.0 * cc * double(c->L.V) * nrhs;
    }
    return lp_check_err(c);
}

int dwf_lp_set_variant(dwf_ctx* c, int variant)
{
    if (!c || !c->lp || variant < -1 || variant > 1)
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_set_variant: bad variant or no network") : DWF_BAD_ARG;
    c->lp->variant = variant;
    return DWF_OK;
}

int dwf_lp_set_krylov(dwf_ctx* c, int method, int restart)
{
    if (!c || !c->lp || method < 0 || method > 1 ||
        (method == 0 && (restart < 4 || restart > kGcrMax || restart % 4 != 0)))
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_set_krylov: bad method or restart length, or no network")
                 : DWF_BAD_ARG;
    c->lp->krylov = method;
    if (method == 0)
        c->lp->gcr_m = restart;
    return DWF_OK;
}

int dwf_lp_set_solver(dwf_ctx* c, double inner_tol, int inner_maxiter, int outer_max)
{
    if (!c || !c->lp || !(inner_tol > 0.0 && inner_tol < 1.0) || inner_maxiter < 1 || outer_max < 1)
        return c ? ctx_fail(c, DWF_BAD_ARG, "dwf_lp_set_solver: bad arguments or no network") : DWF_BAD_ARG;
    c->lp->inner_tol = inner_tol;
    c->lp->inner_max = inner_maxiter;
    c->lp->outer_max = outer_max;
    return DWF_OK;
}

}  // extern "C"
