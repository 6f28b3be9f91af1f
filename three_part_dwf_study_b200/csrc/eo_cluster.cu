// Even-odd Schur mixed CG with one thread-block cluster per right-hand side
// and the FP32 Krylov fields resident in the cluster's shared memory.
//
// The grid-wide kernel (cg_eo_mixed_kernel) runs every right-hand side of a
// batch in lock step: five grid barriers per iteration across all blocks, the
// FP32 fields (p, r, e, t, y: ~15 MB per right-hand side-batch each) streaming
// through L2. Here a cluster of CS CTAs (one per SM) owns one right-hand side
// at a time: CTA c holds time rows [c R, (c+1) R) (R = Nt / CS) of every field
// for every fifth-dimension slice in its own shared memory, the stencil reads
// the rows t0 - 1 and t0 + R of its neighbours through distributed shared
// memory, and the phases are separated by cluster barriers only. Right-hand
// sides are independent, so clusters never wait for one another; each takes
// the right-hand sides cluster_id, cluster_id + nclusters, ...
//
// Per iteration (FP32; the same algebra as cg_eo_mixed_kernel):
//   P1 (4-D even sites)  y = M5^-1 H_eo p        four lanes per 4-D site
//   P2 (5-D odd sites)   t = M5 p - H_oe y, |t|^2              | cluster barrier
//   P3 (4-D even sites)  y = M5^dag^-1 H^dag_eo t               | cluster barrier
//   P4 (5-D odd sites)   Ap = M5^dag t - H^dag_oe y; e += alpha p; r -= alpha Ap, |r|^2
//   P5 (5-D odd sites)   p = r + beta p                         | cluster barrier
// Reliable updates (FP64, fields x, b, t64, y64 in global memory) recompute the
// residual of the Schur normal equation from x + e when the FP32 residual has
// fallen by delta^2 since the last one, or convergence is in sight.
//
// M5^-1 (per spin an Ls x Ls bidiagonal matrix with the m_f corner, closed
// form in eo.cuh) is applied by four lanes per 4-D site, each holding Ls/4
// consecutive slices: the two fifth-dimension recurrences become a suffix and
// a prefix sum with geometric weights c^-k (c = 3 - M5 >= 1), scanned across
// the four lanes with shuffles.
#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "context.cuh"
#include "eo.cuh"
#include "persist.cuh"

namespace cg = cooperative_groups;

namespace dwfb {

namespace {

constexpr int kClThreads = 512;
constexpr int kClMaxLs = 32;

// Cluster layout: CTA `rank` holds rows t in [rank R, rank R + R) of each
// parity field; element (s, t, k) (k = x / 2) at local (s R + t - rank R) Nxh + k.
struct ClGeo
{
    int Nt, Nx, Nxh, Vh, Ls, R, CS;
    int n4;  // 4-D sites of one parity per CTA: R Nxh
    int n5;  // 5-D sites of one parity per CTA: Ls R Nxh
};

// Compile-time part of the geometry: rows per CTA, x sites per parity row,
// slices per lane (Ls = 4 L4). The kernel is instantiated for the shapes the
// study uses (launch_eo_cluster lists them); integer index arithmetic on them
// folds to shifts and constants.
template <int R_, int NXH_, int L4_>
struct ClShape
{
    static constexpr int R = R_, Nxh = NXH_, L4 = L4_, Ls = 4 * L4_;
    static constexpr int n4 = R * Nxh;   // 4-D sites of one parity per CTA
    static constexpr int n5 = Ls * n4;   // 5-D sites of one parity per CTA
    static constexpr int Nx = 2 * Nxh;
};

struct ClDesc
{
    ClGeo G;
    float pw32[kClMaxLs + 1];   // c^-k, k = 0 .. Ls
    double pw64[kClMaxLs + 1];
    double delta;               // reliable-update trigger
};

__device__ __forceinline__ Spinor<float> f4s(float4 v)
{
    return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ float4 s2f4(const Spinor<float>& v)
{
    return make_float4(v.s0.x, v.s0.y, v.s1.x, v.s1.y);
}

// Loader of a cluster FP32 field at (s, t, k): rows [t0, t0 + R) from this
// CTA's own part, the two neighbouring rows t0 - 1 and t0 + R (the only other
// rows a hop reads) from a halo buffer of this CTA, into which the neighbouring
// CTAs stored those rows while they computed them (halo_push).
struct ClRows
{
    const float4* halo;  // [2][Ls][Nxh]: row t0 - 1, row t0 + R
    int t0;
    int tm;              // row t0 - 1, wrapped: halo slot 0; the other outside row is slot 1
};

template <class S>
struct ClLd
{
    const float4* base;
    const ClRows* w;
    __device__ __forceinline__ Spinor<float> sp(int s, int t, int k) const
    {
        const int tl = t - w->t0;
        if (tl >= 0 && tl < S::R)
            return f4s(base[(s * S::R + tl) * S::Nxh + k]);
        const int slot = (t == w->tm) ? 0 : 1;
        return f4s(w->halo[(slot * S::Ls + s) * S::Nxh + k]);
    }
};

// Halo exchange by remote stores: the CTA that computes a value of its first
// row (tl = 0) also stores it into slot 1 of the halo buffer of CTA rank - 1
// (whose row t0 + R it is), a value of its last row (tl = R - 1) into slot 0
// of CTA rank + 1's. The stores need no wait of their own: the cluster barrier
// that ends the phase makes them visible. Two halo buffers alternate so that a
// phase reads one while its stores fill the other.
template <class S>
struct HaloPush
{
    float4* prev;  // halo buffer `dst` of CTA rank - 1 (generic address in the cluster)
    float4* next;  // of CTA rank + 1
    __device__ __forceinline__ void put(int s, int tl, int k, float4 v) const
    {
        if (tl == 0)
            prev[(S::Ls + s) * S::Nxh + k] = v;   // slot 1
        if (tl == S::R - 1)
            next[s * S::Nxh + k] = v;             // slot 0
    }
};

template <class S>
__device__ __forceinline__ HaloPush<S> halo_to(float4* dst, int CS, int rank)
{
    cg::cluster_group cl = cg::this_cluster();
    return {cl.map_shared_rank(dst, (rank + CS - 1) % CS), cl.map_shared_rank(dst, (rank + 1) % CS)};
}

// Loader of a global FP64 parity field (s Vh + t Nxh + k).
template <class S>
struct GlLd
{
    const double2* __restrict__ f;
    int Vh;
    __device__ __forceinline__ Spinor<double> sp(int s, int t, int k) const
    {
        return ld_spinor(f, long(s) * Vh + t * S::Nxh + k);
    }
};

// x (global FP64) + e (cluster FP32).
template <class S>
struct XeLd
{
    const double2* __restrict__ x;
    ClLd<S> e;
    int Vh;
    __device__ __forceinline__ Spinor<double> sp(int s, int t, int k) const
    {
        const Spinor<double> a = ld_spinor(x, long(s) * Vh + t * S::Nxh + k);
        const Spinor<float> b = e.sp(s, t, k);
        return {mkc(a.s0.x + double(b.s0.x), a.s0.y + double(b.s0.y)),
                mkc(a.s1.x + double(b.s1.x), a.s1.y + double(b.s1.y))};
    }
};

// Hop term H (H^dag when DAG) at (s, t, x) of the other parity's field read
// through `ld` (eo_hop with the cluster layout's addressing).
template <bool DAG, typename R, class S, typename LD>
__device__ __forceinline__ Spinor<R> cl_hop(const LD& ld, const cplx<R>* __restrict__ U, const Lat& L,
                                            int Nt, int s, int t, int x)
{
    constexpr int Nx = S::Nx;
    const int tp = (t + 1 == Nt) ? 0 : t + 1;
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const Spinor<R> vtp = ld.sp(s, tp, x >> 1);
    const Spinor<R> vtm = ld.sp(s, tm, x >> 1);
    const Spinor<R> vxp = ld.sp(s, t, xp >> 1);
    const Spinor<R> vxm = ld.sp(s, t, xm >> 1);
    const int here = t * Nx + x;
    const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
    const R stm = (t == 0) ? R(L.bct) : R(1);
    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    cplx<R> up, lo;
    hop4<DAG, R>(vtp, vtm, vxp, vxm, U[here], U[tm * Nx + x], U[L.V + here], U[L.V + t * Nx + xm], stp,
                 stm, sxp, sxm, up, lo);
    return {R(-0.5) * up, R(-0.5) * lo};
}

// M5 (M5^dag when DAG) at (s, t, k) of an odd field read through `ld`
// (eo_m5 with the cluster layout's addressing).
template <bool DAG, typename R, typename LD>
__device__ __forceinline__ Spinor<R> cl_m5(const LD& ld, const Lat& L, int Ls, int s, int t, int k)
{
    const Spinor<R> c = ld.sp(s, t, k);
    const R dg = R(L.diag);
    Spinor<R> o{dg * c.s0, dg * c.s1};
    const int sup = (s + 1 == Ls) ? 0 : s + 1;
    const R cup = (s + 1 == Ls) ? R(L.mf) : R(-1);
    const int sdn = (s == 0) ? Ls - 1 : s - 1;
    const R cdn = (s == 0) ? R(L.mf) : R(-1);
    if (!DAG)
    {
        o.s1 += cup * ld.sp(sup, t, k).s1;
        o.s0 += cdn * ld.sp(sdn, t, k).s0;
    }
    else
    {
        o.s1 += cdn * ld.sp(sdn, t, k).s1;
        o.s0 += cup * ld.sp(sup, t, k).s0;
    }
    return o;
}

#define DWFB_SHFL_CPLX(T)                                                                        \
    __device__ __forceinline__ T shfl_c(T v, int src, int width)                               \
    {                                                                                          \
        return mkc(__shfl_sync(0xffffffffu, v.x, src, width),                                  \
                   __shfl_sync(0xffffffffu, v.y, src, width));                                 \
    }                                                                                          \
    __device__ __forceinline__ T shfl_dn(T v, int d, int width)                                \
    {                                                                                          \
        return mkc(__shfl_down_sync(0xffffffffu, v.x, d, width),                               \
                   __shfl_down_sync(0xffffffffu, v.y, d, width));                              \
    }                                                                                          \
    __device__ __forceinline__ T shfl_up(T v, int d, int width)                                \
    {                                                                                          \
        return mkc(__shfl_up_sync(0xffffffffu, v.x, d, width),                                 \
                   __shfl_up_sync(0xffffffffu, v.y, d, width));                                \
    }
DWFB_SHFL_CPLX(float2)
DWFB_SHFL_CPLX(double2)
#undef DWFB_SHFL_CPLX

// y = M5^-1 z (M5^dag^-1 when DAG) for one 4-D site, the Ls slices spread over
// the four lanes q of a lane group (lane q holds z[j], s = q L4 + j). Up form
// (spin DAG ? 0 : 1): y(s) = U(s) - m_f y0 c^-(Ls-s), U(s) = sum_{k>=s} z(k)
// c^-(k-s+1), y0 = U(0) / (1 + m_f c^-Ls). Down form (the other spin):
// y(s) = D(s) - m_f yL c^-(s+1), D(s) = sum_{k<=s} z(k) c^-(s-k+1),
// yL = D(Ls-1) / (1 + m_f c^-Ls). All lanes of the warp take part.
template <bool DAG, typename R, int L4>
__device__ __forceinline__ void cl_m5inv(Spinor<R> (&z)[L4], int q, const R* pw, int Ls, R mf)
{
    using T = cplx<R>;
    const R ci = pw[1];
    // this lane's block totals: T_q = sum_j z_up(j) c^-(j+1) (= U restricted to
    // the block, at its first slice) and T'_q = sum_j z_dn(j) c^-(L4-j)
    T Tu = mkc(R(0), R(0)), Td = mkc(R(0), R(0));
#pragma unroll
    for (int j = L4 - 1; j >= 0; --j)
        Tu = ci * ((DAG ? z[j].s0 : z[j].s1) + Tu);
#pragma unroll
    for (int j = 0; j < L4; ++j)
        Td = ci * ((DAG ? z[j].s1 : z[j].s0) + Td);
    const R cL4 = pw[L4];
    // suffix scan over lanes of the block totals: B_q = sum_{j>=q} c^-(L4 (j-q)) T_j
    T B = Tu;
    {
        T o = shfl_dn(B, 1, 4);
        B = (q + 1 < 4) ? B + cL4 * o : B;
        o = shfl_dn(B, 2, 4);
        B = (q + 2 < 4) ? B + (cL4 * cL4) * o : B;
    }
    // prefix scan: E_q = sum_{j<=q} c^-(L4 (q-j)) T'_j
    T E = Td;
    {
        T o = shfl_up(E, 1, 4);
        E = (q >= 1) ? E + cL4 * o : E;
        o = shfl_up(E, 2, 4);
        E = (q >= 2) ? E + (cL4 * cL4) * o : E;
    }
    T carry_u = shfl_dn(B, 1, 4);
    carry_u = (q + 1 < 4) ? carry_u : mkc(R(0), R(0));
    T carry_d = shfl_up(E, 1, 4);
    carry_d = (q >= 1) ? carry_d : mkc(R(0), R(0));
    const int lane0 = (threadIdx.x & 31) & ~3;
    const T S = shfl_c(B, lane0, 32);       // U(0), from lane 0 of the group
    const T Sp = shfl_c(E, lane0 + 3, 32);  // D(Ls-1), from lane 3
    const R den = R(1) / (R(1) + mf * pw[Ls]);
    const T y0 = den * S, yL = den * Sp;
    const int a = q * L4;
    // up form, in place, downwards: U(s) = U_loc(s) + c^-(L4-j) B_{q+1}
    T u = mkc(R(0), R(0));
#pragma unroll
    for (int j = L4 - 1; j >= 0; --j)
    {
        u = ci * ((DAG ? z[j].s0 : z[j].s1) + u);
        const T yv = u + pw[L4 - j] * carry_u - (mf * pw[Ls - a - j]) * y0;
        if (DAG)
            z[j].s0 = yv;
        else
            z[j].s1 = yv;
    }
    // down form, in place, upwards: D(s) = D_loc(s) + c^-(j+1) E_{q-1}
    T dn = mkc(R(0), R(0));
#pragma unroll
    for (int j = 0; j < L4; ++j)
    {
        dn = ci * ((DAG ? z[j].s1 : z[j].s0) + dn);
        const T yv = dn + pw[j + 1] * carry_d - (mf * pw[a + j + 1]) * yL;
        if (DAG)
            z[j].s1 = yv;
        else
            z[j].s0 = yv;
    }
}

// Deterministic sum over the cluster of one value per CTA: every CTA writes
// its block sum to red[slot] (own shared memory); after the cluster barrier
// thread r fetches CTA r's entry into gath[r] and every thread sums gath in
// rank order, so all CTAs hold the same bits.
__device__ __forceinline__ double cl_gather(double* red, double* gath, int slot, int CS)
{
    if (threadIdx.x < CS)
        gath[threadIdx.x] = *cg::this_cluster().map_shared_rank(red + slot, threadIdx.x);
    __syncthreads();
    double v = 0.0;
    for (int r = 0; r < CS; ++r)
        v += gath[r];
    __syncthreads();
    return v;
}

// Cluster barrier (release / acquire at cluster scope): shared memory written
// before it by any CTA of the cluster is visible to all after it.
__device__ __forceinline__ void cl_sync() { cg::this_cluster().sync(); }

// The same after phases that write global memory (the FP64 reliable-update
// fields), with a device-scope fence ahead of the barrier.
__device__ __forceinline__ void cl_sync_global()
{
    __threadfence();
    cg::this_cluster().sync();
}

}  // namespace

// A thread's 4-D site in one of the FP32 phases, fixed for the whole solve:
// where its four hop neighbours sit (slice 0) in the other parity's field.
// The t neighbours are in this CTA's part (slice stride R Nxh) or in a halo
// buffer (slice stride Nxh); the x neighbours are always in the own part.
struct ClNbr
{
    int tp, tm;          // offsets of the t+1, t-1 neighbours at slice 0
    bool tp_own, tm_own;
    int xp, xm;          // own-part offsets of the x+1, x-1 neighbours at slice 0
};

template <class S>
__device__ __forceinline__ ClNbr cl_nbr(int tl, int x)
{
    ClNbr n;
    n.tp_own = tl + 1 < S::R;
    n.tp = n.tp_own ? (tl + 1) * S::Nxh + (x >> 1) : S::Ls * S::Nxh + (x >> 1);
    n.tm_own = tl >= 1;
    n.tm = n.tm_own ? (tl - 1) * S::Nxh + (x >> 1) : (x >> 1);
    const int xp = (x + 1 == S::Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? S::Nx - 1 : x - 1;
    n.xp = tl * S::Nxh + (xp >> 1);
    n.xm = tl * S::Nxh + (xm >> 1);
    return n;
}

// The four link phases of the hops from (t, x), FP32, boundary signs folded in
// (exact: the signs are +-1).
struct ClLinks
{
    float2 t, tm, x, xm;
};

__device__ __forceinline__ ClLinks cl_links(const float2* __restrict__ U, const Lat& L, int Nt, int Nx,
                                            int t, int x)
{
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const float stp = (t == Nt - 1) ? float(L.bct) : 1.f;
    const float stm = (t == 0) ? float(L.bct) : 1.f;
    const float sxp = (x == Nx - 1) ? float(L.bcx) : 1.f;
    const float sxm = (x == 0) ? float(L.bcx) : 1.f;
    return {stp * U[t * Nx + x], stm * U[tm * Nx + x], sxp * U[L.V + t * Nx + x], sxm * U[L.V + t * Nx + xm]};
}

// Hop term at slice s from precomputed neighbours and links (cl_hop for the
// FP32 phases): own = the other parity field's own part, halo = its halo buffer.
template <bool DAG, class S>
__device__ __forceinline__ Spinor<float> cl_hop_pre(const float4* own, const float4* halo, const ClNbr& n,
                                                    const ClLinks& u, int s)
{
    const float4 a = n.tp_own ? own[n.tp + s * S::n4] : halo[n.tp + s * S::Nxh];
    const float4 b = n.tm_own ? own[n.tm + s * S::n4] : halo[n.tm + s * S::Nxh];
    const float4 c = own[n.xp + s * S::n4];
    const float4 d = own[n.xm + s * S::n4];
    float2 up, lo;
    hop4<DAG, float>(f4s(a), f4s(b), f4s(c), f4s(d), u.t, u.tm, u.x, u.xm, 1.f, 1.f, 1.f, 1.f, up, lo);
    return {-0.5f * up, -0.5f * lo};
}

// M5 (M5^dag when DAG) at slice s of the own 4-D site h of an odd field.
template <bool DAG, class S>
__device__ __forceinline__ Spinor<float> cl_m5_pre(const float4* f, const Lat& L, int s, int h)
{
    const Spinor<float> c = f4s(f[s * S::n4 + h]);
    const float dg = float(L.diag);
    Spinor<float> o{dg * c.s0, dg * c.s1};
    const int sup = (s + 1 == S::Ls) ? 0 : s + 1;
    const float cup = (s + 1 == S::Ls) ? float(L.mf) : -1.f;
    const int sdn = (s == 0) ? S::Ls - 1 : s - 1;
    const float cdn = (s == 0) ? float(L.mf) : -1.f;
    if (!DAG)
    {
        o.s1 += cup * f4s(f[sup * S::n4 + h]).s1;
        o.s0 += cdn * f4s(f[sdn * S::n4 + h]).s0;
    }
    else
    {
        o.s1 += cdn * f4s(f[sdn * S::n4 + h]).s1;
        o.s0 += cup * f4s(f[sup * S::n4 + h]).s0;
    }
    return o;
}

// Phase timer of cluster 0, rank 0, thread 0 (only when a phase buffer is
// given; the same slots as the grid-wide kernel's).
__device__ __forceinline__ void cl_mark(unsigned long long* ph, int k, unsigned long long& t)
{
    if (ph && blockIdx.x == 0 && threadIdx.x == 0)
    {
        const unsigned long long n = globaltimer_ns();
        ph[k] += n - t;
        ph[8 + k] += 1;
        t = n;
    }
}

template <class S>
__global__ void __launch_bounds__(kClThreads, 1) cg_eo_cluster_kernel(EoDesc e, ClDesc c)
{
    constexpr int L4 = S::L4;
    const SolveDesc& d = e.d;
    const ClGeo G = c.G;
    const Lat& L = d.L;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = int(cluster.block_rank());
    const int cid = int(blockIdx.x) / G.CS;
    const int ncl = int(gridDim.x) / G.CS;
    extern __shared__ __align__(16) unsigned char cl_smem[];
    float4* Pf = reinterpret_cast<float4*>(cl_smem);
    float4* Rf = Pf + S::n5;
    float4* Ef = Rf + S::n5;
    float4* Tf = Ef + S::n5;
    float4* Yf = Tf + S::n5;
    float4* HA = Yf + S::n5;                     // halo buffers [2][Ls][Nxh] (rows t0 - 1, t0 + R)
    float4* HB = HA + 2 * S::Ls * S::Nxh;
    double* red = reinterpret_cast<double*>(HB + 2 * S::Ls * S::Nxh);   // [8] per-CTA partials
    double* scratch = red + 8;                            // [32] block_sum scratch
    __shared__ double gath[16];
    __shared__ float pw32[kClMaxLs + 1];
    __shared__ double pw64[kClMaxLs + 1];
    for (int k = threadIdx.x; k <= S::Ls; k += blockDim.x)
    {
        pw32[k] = c.pw32[k];
        pw64[k] = c.pw64[k];
    }
    __syncthreads();
    const int t0 = rank * S::R;
    // halo buffer A carries p (read in P1), t (P3) and e (reliable update);
    // B carries y (P2, P4)
    const ClRows rowsA{HA, t0, (t0 + G.Nt - 1) % G.Nt}, rowsB{HB, t0, (t0 + G.Nt - 1) % G.Nt};
    const ClLd<S> P{Pf, &rowsA}, E{Ef, &rowsA}, Tl{Tf, &rowsA}, Y{Yf, &rowsB};
    const HaloPush<S> pushA = halo_to<S>(HA, G.CS, rank), pushB = halo_to<S>(HB, G.CS, rank);
    // thread roles of the FP32 phases, fixed for the solve: in the 4-D phases
    // lanes 4h .. 4h+3 take even 4-D site h (lane q: slices q L4 .. q L4 + L4 - 1);
    // in the 5-D phases thread h + g n4 takes odd 4-D site h and the slices
    // g, g + G4, ... (G4 = threads / n4 slice groups)
    static_assert(4 * S::n4 <= kClThreads, "one 4-D site per lane group");
    constexpr int G4 = kClThreads / S::n4;
    const int eh = threadIdx.x >> 2;
    const bool e_on = eh < S::n4;
    const int etl = e_on ? eh / S::Nxh : 0, ek = e_on ? eh - etl * S::Nxh : 0;
    const int et = t0 + etl, ex = 2 * ek + (et & 1);
    const ClNbr enb = cl_nbr<S>(etl, ex);
    const int oh = threadIdx.x % S::n4, og = threadIdx.x / S::n4;
    const bool o_on = og < G4;
    const int otl = oh / S::Nxh, ok = oh - otl * S::Nxh;
    const int ot = t0 + otl, ox = 2 * ok + ((ot + 1) & 1);
    const ClNbr onb = cl_nbr<S>(otl, ox);
    const long fh = d.fsz;  // complex entries of one global parity field
    const int q = threadIdx.x & 3;

    for (int j = cid; j < d.nrhs; j += ncl)
    {
        const long uo = long(d.rhs_conf[j]) * d.usz;
        const float2* U32 = d.U32 + uo;
        const double2* U64 = d.U64 + uo;
        const double2* bj = d.b + j * fh;
        double2* xj = d.x + j * fh;
        double2* t64 = d.t + j * fh;
        double2* y64 = e.y64 + j * fh;
        const ClLinks eu = cl_links(U32, L, G.Nt, S::Nx, et, ex);
        const ClLinks ou = cl_links(U32, L, G.Nt, S::Nx, ot, ox);
        // ---- x = 0: r = b, r32 = p32 = r, e32 = 0; |b|^2 ----
        double a0 = 0.0;
        for (int l = threadIdx.x; l < S::n5; l += kClThreads)
        {
            const int s = l / S::n4, rem = l - s * S::n4, tl = rem / S::Nxh, k = rem - tl * S::Nxh;
            const Spinor<double> b = ld_spinor(bj, long(s) * G.Vh + (t0 + tl) * S::Nxh + k);
            const float4 r32 = s2f4(persist::to32(b));
            Rf[l] = r32;
            Pf[l] = r32;
            pushA.put(s, tl, k, r32);
            Ef[l] = make_float4(0.f, 0.f, 0.f, 0.f);
            a0 += spinor_norm2(b);
        }
        a0 = block_sum(a0, scratch);
        if (threadIdx.x == 0)
            red[0] = a0;
        cl_sync();
        const double bb = cl_gather(red, gath, 0, G.CS);
        double rr = bb, rru = bb;
        int iters = 0, ru = 0, stalls = 0;
        int state = (bb == 0.0 || persist::converged_now(d, rr, bb)) ? DWF_OK : RHS_ACTIVE;

        unsigned long long ph_t = globaltimer_ns();
        for (int it = 1; it <= d.maxiter && state == RHS_ACTIVE; ++it)
        {
            // P1: y = M5^-1 H_eo p (four lanes per even 4-D site)
            {
                Spinor<float> z[L4];
#pragma unroll
                for (int jj = 0; jj < L4; ++jj)
                    z[jj] = e_on ? cl_hop_pre<false, S>(Pf, HA, enb, eu, q * L4 + jj) : Spinor<float>{};
                cl_m5inv<false, float, L4>(z, q, pw32, S::Ls, float(L.mf));
                if (e_on)
#pragma unroll
                    for (int jj = 0; jj < L4; ++jj)
                    {
                        const float4 v = s2f4(z[jj]);
                        Yf[(q * L4 + jj) * S::n4 + eh] = v;
                        pushB.put(q * L4 + jj, etl, ek, v);
                    }
            }
            cl_sync();
            cl_mark(e.phase_ns, 0, ph_t);
            // P2: t = M5 p - H_oe y, |t|^2
            a0 = 0.0;
            if (o_on)
                for (int sl = og; sl < S::Ls; sl += G4)
                {
                    const Spinor<float> m = cl_m5_pre<false, S>(Pf, L, sl, oh);
                    const Spinor<float> hy = cl_hop_pre<false, S>(Yf, HB, onb, ou, sl);
                    const Spinor<float> v{m.s0 - hy.s0, m.s1 - hy.s1};
                    const float4 v4 = s2f4(v);
                    Tf[sl * S::n4 + oh] = v4;
                    pushA.put(sl, otl, ok, v4);
                    a0 += spinor_norm2(v);
                }
            a0 = block_sum(a0, scratch);
            if (threadIdx.x == 0)
                red[1] = a0;
            cl_sync();
            cl_mark(e.phase_ns, 1, ph_t);
            const double tt = cl_gather(red, gath, 1, G.CS);
            if (tt == 0.0 || !isfinite(tt))
            {
                state = DWF_NOT_CONVERGED;
                iters = it;
                break;
            }
            const float al = float(rr / tt);
            cl_mark(e.phase_ns, 2, ph_t);
            // P3: y = M5^dag^-1 H^dag_eo t
            {
                Spinor<float> z[L4];
#pragma unroll
                for (int jj = 0; jj < L4; ++jj)
                    z[jj] = e_on ? cl_hop_pre<true, S>(Tf, HA, enb, eu, q * L4 + jj) : Spinor<float>{};
                cl_m5inv<true, float, L4>(z, q, pw32, S::Ls, float(L.mf));
                if (e_on)
#pragma unroll
                    for (int jj = 0; jj < L4; ++jj)
                    {
                        const float4 v = s2f4(z[jj]);
                        Yf[(q * L4 + jj) * S::n4 + eh] = v;
                        pushB.put(q * L4 + jj, etl, ek, v);
                    }
            }
            cl_sync();
            cl_mark(e.phase_ns, 3, ph_t);
            // P4: Ap = M5^dag t - H^dag_oe y; e += alpha p; r -= alpha Ap; |r|^2
            a0 = 0.0;
            if (o_on)
                for (int sl = og; sl < S::Ls; sl += G4)
                {
                    const int l = sl * S::n4 + oh;
                    const Spinor<float> m = cl_m5_pre<true, S>(Tf, L, sl, oh);
                    const Spinor<float> hy = cl_hop_pre<true, S>(Yf, HB, onb, ou, sl);
                    const Spinor<float> ap{m.s0 - hy.s0, m.s1 - hy.s1};
                    const Spinor<float> p = f4s(Pf[l]);
                    const float4 en = s2f4(persist::axpy(al, p, f4s(Ef[l])));
                    Ef[l] = en;
                    pushA.put(sl, otl, ok, en);
                    const Spinor<float> rn = persist::axpy(-al, ap, f4s(Rf[l]));
                    Rf[l] = s2f4(rn);
                    a0 += spinor_norm2(rn);
                }
            a0 = block_sum(a0, scratch);
            if (threadIdx.x == 0)
                red[2] = a0;
            cl_sync();
            cl_mark(e.phase_ns, 4, ph_t);
            const double rn = cl_gather(red, gath, 2, G.CS);
            iters = it;
            const bool want = rn < c.delta * c.delta * rru || persist::converged_now(d, rn, bb) ||
                              it == d.maxiter;
            double cf = rn / rr;
            rr = rn;
            if (want)
            {
                // ---- reliable update in FP64: r = b - Dhat^dag Dhat (x + e) ----
                const XeLd<S> xe{xj, E, G.Vh};
                // (a) y64 = M5^-1 H_eo (x + e)
                for (int w = threadIdx.x; w < 4 * S::n4 + ((4 * S::n4) % 32 ? 32 - (4 * S::n4) % 32 : 0);
                     w += kClThreads)
                {
                    const int h = w >> 2;
                    const bool on = h < S::n4;
                    const int tl = on ? h / S::Nxh : 0, k = on ? h - tl * S::Nxh : 0;
                    const int t = t0 + tl, x = 2 * k + (t & 1);
                    Spinor<double> z[L4];
#pragma unroll
                    for (int jj = 0; jj < L4; ++jj)
                        z[jj] = on ? cl_hop<false, double, S>(xe, U64, L, G.Nt, q * L4 + jj, t, x) : Spinor<double>{};
                    cl_m5inv<false, double, L4>(z, q, pw64, S::Ls, L.mf);
                    if (on)
#pragma unroll
                        for (int jj = 0; jj < L4; ++jj)
                            st_spinor(y64, long(q * L4 + jj) * G.Vh + t * S::Nxh + k, z[jj]);
                }
                cl_sync_global();
                // (b) t64 = M5 (x + e) - H_oe y64
                const GlLd<S> yl{y64, G.Vh};
                for (int l = threadIdx.x; l < S::n5; l += kClThreads)
                {
                    const int s = l / S::n4, rem = l - s * S::n4, tl = rem / S::Nxh, k = rem - tl * S::Nxh;
                    const int t = t0 + tl, x = 2 * k + ((t + 1) & 1);
                    const Spinor<double> m = cl_m5<false, double>(xe, L, S::Ls, s, t, k);
                    const Spinor<double> hy = cl_hop<false, double, S>(yl, U64, L, G.Nt, s, t, x);
                    st_spinor(t64, long(s) * G.Vh + t * S::Nxh + k, Spinor<double>{m.s0 - hy.s0, m.s1 - hy.s1});
                }
                cl_sync_global();
                // (c) y64 = M5^dag^-1 H^dag_eo t64
                const GlLd<S> tlg{t64, G.Vh};
                for (int w = threadIdx.x; w < 4 * S::n4 + ((4 * S::n4) % 32 ? 32 - (4 * S::n4) % 32 : 0);
                     w += kClThreads)
                {
                    const int h = w >> 2;
                    const bool on = h < S::n4;
                    const int tl = on ? h / S::Nxh : 0, k = on ? h - tl * S::Nxh : 0;
                    const int t = t0 + tl, x = 2 * k + (t & 1);
                    Spinor<double> z[L4];
#pragma unroll
                    for (int jj = 0; jj < L4; ++jj)
                        z[jj] = on ? cl_hop<true, double, S>(tlg, U64, L, G.Nt, q * L4 + jj, t, x) : Spinor<double>{};
                    cl_m5inv<true, double, L4>(z, q, pw64, S::Ls, L.mf);
                    if (on)
#pragma unroll
                        for (int jj = 0; jj < L4; ++jj)
                            st_spinor(y64, long(q * L4 + jj) * G.Vh + t * S::Nxh + k, z[jj]);
                }
                cl_sync_global();
                // (d) r = b - (M5^dag t64 - H^dag_oe y64); x += e; r32 = r; e = 0
                a0 = 0.0;
                for (int l = threadIdx.x; l < S::n5; l += kClThreads)
                {
                    const int s = l / S::n4, rem = l - s * S::n4, tl = rem / S::Nxh, k = rem - tl * S::Nxh;
                    const int t = t0 + tl, x = 2 * k + ((t + 1) & 1);
                    const long gi = long(s) * G.Vh + t * S::Nxh + k;
                    const Spinor<double> m = cl_m5<true, double>(tlg, L, S::Ls, s, t, k);
                    const Spinor<double> hy = cl_hop<true, double, S>(yl, U64, L, G.Nt, s, t, x);
                    const Spinor<double> b = ld_spinor(bj, gi);
                    const Spinor<double> r{b.s0 - (m.s0 - hy.s0), b.s1 - (m.s1 - hy.s1)};
                    const Spinor<double> xo = ld_spinor(xj, gi);
                    const Spinor<float> ev = f4s(Ef[l]);
                    st_spinor(xj, gi, Spinor<double>{mkc(xo.s0.x + double(ev.s0.x), xo.s0.y + double(ev.s0.y)),
                                                     mkc(xo.s1.x + double(ev.s1.x), xo.s1.y + double(ev.s1.y))});
                    Rf[l] = s2f4(persist::to32(r));
                    Ef[l] = make_float4(0.f, 0.f, 0.f, 0.f);
                    a0 += spinor_norm2(r);
                }
                a0 = block_sum(a0, scratch);
                if (threadIdx.x == 0)
                    red[3] = a0;
                cl_sync_global();
                const double rt = cl_gather(red, gath, 3, G.CS);
                ru += 1;
                cf = cf * (rt / rr);
                stalls = (rt >= 0.5 * rru) ? stalls + 1 : 0;
                rr = rt;
                rru = rt;
                if (persist::converged_now(d, rt, bb))
                    state = DWF_OK;
                else if (!isfinite(rt) || stalls >= d.stall_limit || it == d.maxiter)
                    state = DWF_NOT_CONVERGED;
                if (state != RHS_ACTIVE)
                    break;
            }
            cl_mark(e.phase_ns, 5, ph_t);
            // P5: p = r + beta p
            const float beta = float(cf);
            if (o_on)
                for (int sl = og; sl < S::Ls; sl += G4)
                {
                    const int l = sl * S::n4 + oh;
                    const float4 v = s2f4(persist::axpy(beta, f4s(Pf[l]), f4s(Rf[l])));
                    Pf[l] = v;
                    pushA.put(sl, otl, ok, v);
                }
            cl_sync();
            cl_mark(e.phase_ns, 6, ph_t);
        }
        if (rank == 0 && threadIdx.x == 0)
        {
            d.out_iters[j] = iters;
            d.out_status[j] = state == RHS_ACTIVE ? DWF_NOT_CONVERGED : state;
            d.out_relres[j] = bb > 0.0 ? sqrt(rr / bb) : 0.0;
            d.out_ru[j] = ru;
        }
        // the next right-hand side overwrites the fields and partials
        cl_sync();
    }
}

// shapes: 64x64x16 (16-CTA clusters), 64x32x16 and 32x32x16 (8-CTA),
// 64x56x16 (16-CTA), 32x16x24 (8-CTA)
#define DWFB_CL_SHAPES(X) X(4, 32, 4) X(8, 16, 4) X(4, 16, 4) X(4, 28, 4) X(4, 8, 6)
#define DWFB_CL_INST(r, h, l) template __global__ void cg_eo_cluster_kernel<ClShape<r, h, l>>(EoDesc, ClDesc);
DWFB_CL_SHAPES(DWFB_CL_INST)
#undef DWFB_CL_INST

// Launch the cluster solver for a batch prepared by propagators_eo (fields in
// EoDesc as for cg_eo_mixed_kernel). Returns DWF_BAD_ARG (nothing launched)
// when the lattice or the device does not allow it: the caller then runs the
// grid-wide kernel. A dry call only checks, and reports in *wave (when not
// null) how many right-hand sides the resident clusters solve at once.
// Launch shape of the cluster kernel per (device, kernel): attributes set and
// the resident-cluster count queried once, so that a later call (the one a
// stream capture records) issues the launch alone.
struct ClLaunchShape
{
    int nclust = 0;
};

// dry: check that the cluster kernel takes this batch and prepare its launch
// shape without launching (*launched tells whether it would launch).
int launch_eo_cluster(dwf_ctx* c, EoDesc& e, bool* launched, bool dry, int* wave)
{
    static std::map<std::pair<int, const void*>, ClLaunchShape> shapes;
    static std::mutex shapes_mu;
    *launched = false;
    const Lat& L = c->L;
    const int Ls = L.Ls;
    if (Ls % 4 != 0 || Ls > kClMaxLs)
        return DWF_BAD_ARG;
    ClDesc cd{};
    ClGeo& G = cd.G;
    G.Nt = L.Nt;
    G.Nx = L.Nx;
    G.Nxh = L.Nx / 2;
    G.Vh = L.V / 2;
    G.Ls = Ls;
    int CS = 0;
    size_t smem = 0;
    for (int cs : {8, 16})
    {
        if (L.Nt % cs != 0)
            continue;
        const int R = L.Nt / cs;
        const int n5 = Ls * R * G.Nxh;
        const size_t sm = size_t(5) * n5 * sizeof(float4) + size_t(4) * Ls * G.Nxh * sizeof(float4) +
                          40 * sizeof(double);
        // one right-hand side's fields must fit the cluster's shared memory and
        // the lane groups of the 4-D phases must fill whole warps
        if (sm <= size_t(200 * 1024) && (R * G.Nxh) % 8 == 0)
        {
            CS = cs;
            smem = sm;
            G.R = R;
            G.n4 = R * G.Nxh;
            G.n5 = n5;
            break;
        }
    }
    if (CS == 0)
        return DWF_BAD_ARG;
    G.CS = CS;
    const double cc = L.diag;
    double p = 1.0;
    for (int k = 0; k <= Ls; ++k)
    {
        cd.pw64[k] = p;
        cd.pw32[k] = float(p);
        p /= cc;
    }
    cd.delta = e.d.delta;
    const void* fn = nullptr;
#define DWFB_CL_PICK(r, h, l)                                                              \
    if (G.R == r && G.Nxh == h && Ls == 4 * l)                                             \
        fn = reinterpret_cast<const void*>(&cg_eo_cluster_kernel<ClShape<r, h, l>>);
    DWFB_CL_SHAPES(DWFB_CL_PICK)
#undef DWFB_CL_PICK
    if (!fn)
        return DWF_BAD_ARG;
    std::lock_guard<std::mutex> lock(shapes_mu);
    ClLaunchShape& sh = shapes[std::make_pair(c->device, fn)];
    if (sh.nclust == 0 &&
        (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess ||
         (CS > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)))
    {
        cudaGetLastError();
        return DWF_BAD_ARG;
    }
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(CS);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(unsigned(CS * std::max(1, e.d.nrhs)));
    if (sh.nclust == 0)
    {
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, fn, &cfg) != cudaSuccess || nc < 1)
        {
            cudaGetLastError();
            return DWF_BAD_ARG;
        }
        sh.nclust = nc;
    }
    if (dry)
    {
        *launched = true;
        if (wave)
            *wave = sh.nclust;
        return DWF_OK;
    }
    const int nclust = std::min(sh.nclust, e.d.nrhs);
    cfg.gridDim = dim3(unsigned(CS * nclust));
    void* args[] = {&e, &cd};
    if (cudaLaunchKernelExC(&cfg, fn, args) != cudaSuccess)
        return ctx_fail(c, DWF_CUDA_ERROR, "even-odd cluster solver: launch failed");
    *launched = true;
    return DWF_OK;
}

}  // namespace dwfb
