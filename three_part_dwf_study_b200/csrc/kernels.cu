// Non-persistent kernels: link phases, standalone operator application and
// the FP64 true residual.
#include "kernels.cuh"

namespace dwfb {

__global__ void links_kernel(const double* __restrict__ theta, long n, double2* __restrict__ U64,
                             float2* __restrict__ U32)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n;
         i += long(gridDim.x) * blockDim.x)
    {
        double sn, cs;
        sincos(theta[i], &sn, &cs);
        U64[i] = make_double2(cs, sn);
        U32[i] = make_float2(float(cs), float(sn));
    }
}

template <bool DAG, typename R>
__global__ void __launch_bounds__(256)
    dirac_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out, long fsz,
                 const cplx<R>* __restrict__ U, long usz, const int* __restrict__ conf,
                 int conf0)
{
    const int j = blockIdx.y;
    const int c = conf ? conf[j] : conf0;
    const cplx<R>* Uj = U + long(c) * usz;
    const cplx<R>* inj = in + j * fsz;
    cplx<R>* outj = out + j * fsz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.nsite; i += gridDim.x * blockDim.x)
    {
        int s, t, x;
        site_coords(L, i, s, t, x);
        st_spinor(outj, i, dirac_site<DAG, R>(inj, Uj, L, s, t, x));
    }
}

// One thread per 5-D site, warps over 32 consecutive x of one row (Nx a
// multiple of 32), x neighbours by shuffle; the loop is warp-uniform.
template <bool DAG, typename R>
__global__ void __launch_bounds__(256)
    dirac_warp_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out, long fsz,
                      const cplx<R>* __restrict__ U, long usz, const int* __restrict__ conf,
                      int conf0)
{
    const int j = blockIdx.y;
    const int c = conf ? conf[j] : conf0;
    const cplx<R>* Uj = U + long(c) * usz;
    const cplx<R>* inj = in + j * fsz;
    cplx<R>* outj = out + j * fsz;
    const int lane = threadIdx.x & 31;
    // L.nsite is a multiple of 32 (Nx is), so every warp's 32 sites are valid
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < L.nsite;
         base += gridDim.x * blockDim.x)
    {
        const int i = base + lane;
        int s, t, x;
        site_coords(L, i, s, t, x);
        st_spinor(outj, i, dirac_site_warp<DAG, R>(inj, Uj, L, s, t, x, lane));
    }
}

template __global__ void dirac_warp_kernel<false, double>(Lat, const double2*, double2*, long,
                                                          const double2*, long, const int*, int);
template __global__ void dirac_warp_kernel<true, double>(Lat, const double2*, double2*, long,
                                                         const double2*, long, const int*, int);
template __global__ void dirac_warp_kernel<false, float>(Lat, const float2*, float2*, long,
                                                         const float2*, long, const int*, int);
template __global__ void dirac_warp_kernel<true, float>(Lat, const float2*, float2*, long,
                                                        const float2*, long, const int*, int);

template <bool DAG, typename R, int RT>
__global__ void __launch_bounds__(256)
    wilson_rows_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out, long fsz,
                       const cplx<R>* __restrict__ U, long usz, const int* __restrict__ conf,
                       int conf0)
{
    using T = cplx<R>;
    const int j = blockIdx.z;
    const int c = conf ? conf[j] : conf0;
    const T* __restrict__ Uj = U + long(c) * usz;
    const T* __restrict__ inj = in + j * fsz;
    T* __restrict__ outj = out + j * fsz;
    const int Nt = L.Nt, Nx = L.Nx, V = L.V;
    const int lane = threadIdx.x;
    const int t0 = (blockIdx.y * blockDim.y + threadIdx.y) * RT;
    if (t0 >= Nt)
        return;  // the whole warp: t0 is the same for its 32 lanes
    const int x = blockIdx.x * 32 + lane;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;

    // every load up front: rows t0-1 .. t0+RT of this column (t links of
    // rows t0-1 .. t0+RT-1), the x links of the RT rows, and the neighbour
    // outside the warp for the edge lanes (x+1 for lane 31, x-1 and its link
    // for lane 0)
    Spinor<R> v[RT + 2], h[RT] = {};
    T ut[RT + 1], ux[RT], uh[RT] = {};
#pragma unroll
    for (int k = 0; k < RT + 2; ++k)
    {
        int t = t0 - 1 + k;  // in [-1, Nt] since Nt % RT == 0
        t = (t < 0) ? t + Nt : (t >= Nt ? t - Nt : t);
        v[k] = ld_spinor(inj, long(t) * Nx + x);
        if (k <= RT)
            ut[k] = Uj[t * Nx + x];
    }
#pragma unroll
    for (int k = 0; k < RT; ++k)
    {
        const int row = (t0 + k) * Nx;
        ux[k] = Uj[V + row + x];
        if (lane == 31)
            h[k] = ld_spinor(inj, long(row) + xp);
        if (lane == 0)
        {
            h[k] = ld_spinor(inj, long(row) + xm);
            uh[k] = Uj[V + row + xm];
        }
    }

    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    const R dg = R(L.diag);
    const int lp = (lane + 1) & 31, lm = (lane + 31) & 31;
#pragma unroll
    for (int k = 0; k < RT; ++k)
    {
        const int t = t0 + k;
        const Spinor<R>& cc = v[k + 1];
        Spinor<R> vxp{shfl_c(cc.s0, lp), shfl_c(cc.s1, lp)};
        Spinor<R> vxm{shfl_c(cc.s0, lm), shfl_c(cc.s1, lm)};
        T Uxm = shfl_c(ux[k], lm);
        if (lane == 31)
            vxp = h[k];
        if (lane == 0)
        {
            vxm = h[k];
            Uxm = uh[k];
        }
        const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
        const R stm = (t == 0) ? R(L.bct) : R(1);
        T up, lo;
        hop4<DAG, R>(v[k + 2], v[k], vxp, vxm, ut[k + 1], ut[k], ux[k], Uxm, stp, stm, sxp, sxm,
                     up, lo);
        st_spinor(outj, long(t) * Nx + x, Spinor<R>{dg * cc.s0 - R(0.5) * up, dg * cc.s1 - R(0.5) * lo});
    }
}

#define DWFB_WILSON_ROWS(DAG, R)                                                                  \
    template __global__ void wilson_rows_kernel<DAG, R, kWilsonRows>(                             \
        Lat, const cplx<R>*, cplx<R>*, long, const cplx<R>*, long, const int*, int);
DWFB_WILSON_ROWS(false, double)
DWFB_WILSON_ROWS(true, double)
DWFB_WILSON_ROWS(false, float)
DWFB_WILSON_ROWS(true, float)
#undef DWFB_WILSON_ROWS

// One thread per 4-D site, all Ls slices (links and the fifth-dimension
// neighbours reused from registers); blocks are 32 x 8 tiles of (x, t) so the
// t +- 1 neighbours of a warp are mostly loaded by the block's other warps.
template <bool DAG, typename R>
__global__ void __launch_bounds__(256)
    dirac_col_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out, long fsz,
                     const cplx<R>* __restrict__ U, long usz, const int* __restrict__ conf,
                     int conf0)
{
    const int j = blockIdx.z;
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int t = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= L.Nx || t >= L.Nt)
        return;
    const int c = conf ? conf[j] : conf0;
    cplx<R>* outj = out + j * fsz;
    const int here = t * L.Nx + x;
    dirac_column<DAG, R>(in + j * fsz, U + long(c) * usz, L, t, x,
                         [&](int s, const Spinor<R>& o) { st_spinor(outj, long(s) * L.V + here, o); });
}

// Slices of lookahead that dirac_colx_kernel prefetches into L1 (0: none; at
// 512x512x16, 1 / 2 / 3 slices gave 3794 / 4188 / 4108 GB/s in FP64).
#ifndef DWFB_COLX_PREFETCH
#define DWFB_COLX_PREFETCH 2
#endif

__device__ __forceinline__ void prefetch_l1(const void* p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <bool DAG, typename R>
__global__ void __launch_bounds__(256)
    dirac_colx_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out, long fsz,
                      const cplx<R>* __restrict__ U, long usz, const int* __restrict__ conf,
                      int conf0)
{
    using T = cplx<R>;
    const int j = blockIdx.z;
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (t >= L.Nt)
        return;  // the whole warp: t is the same for its 32 lanes
    const int c = conf ? conf[j] : conf0;
    const T* __restrict__ Uj = U + long(c) * usz;
    const T* __restrict__ inj = in + j * fsz;
    T* __restrict__ outj = out + j * fsz;
    const int Nt = L.Nt, Nx = L.Nx, V = L.V, Ls = L.Ls;
    const int x = blockIdx.x * 32 + lane;
    const int tp = (t + 1 == Nt) ? 0 : t + 1;
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const int here = t * Nx + x, itp = tp * Nx + x, itm = tm * Nx + x;
    // the neighbour outside the warp: x+1 for lane 31, x-1 for lane 0
    const int ie = t * Nx + ((lane == 31) ? xp : xm);
    const bool edge = (lane == 0) || (lane == 31);
    const int lp = (lane + 1) & 31, lm = (lane + 31) & 31;

    const T Ut = Uj[here];
    const T Utm = Uj[itm];
    const T Ux = Uj[V + here];
    T Uxm = shfl_c(Ux, lm);
    if (lane == 0)
        Uxm = Uj[V + t * Nx + xm];
    const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
    const R stm = (t == 0) ? R(L.bct) : R(1);
    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    const R dg = R(L.diag), mf = R(L.mf);

    // slice s's operands are loaded one slice ahead, before slice s - 1 is computed
    const Spinor<R> first = ld_spinor(inj, here);
    Spinor<R> prev = L.fifth ? ld_spinor(inj, long(Ls - 1) * V + here) : first;
    Spinor<R> cur = first;
    Spinor<R> vtp = ld_spinor(inj, itp), vtm = ld_spinor(inj, itm), h = {};
    if (edge)
        h = ld_spinor(inj, ie);
    for (int s = 0; s < Ls; ++s)
    {
        if (DWFB_COLX_PREFETCH > 0 && s + DWFB_COLX_PREFETCH < Ls)
        {
            // pull slice s + DWFB_COLX_PREFETCH into L1 without holding registers for it
            const T* const pb = inj + 2 * long(s + DWFB_COLX_PREFETCH) * V;
            prefetch_l1(pb + 2 * here);
            prefetch_l1(pb + 2 * itp);
            prefetch_l1(pb + 2 * itm);
        }
        Spinor<R> nxt = first, ntp = {}, ntm = {}, nh = {};
        if (s + 1 < Ls)
        {
            const long sb = long(s + 1) * V;
            nxt = ld_spinor(inj, sb + here);
            ntp = ld_spinor(inj, sb + itp);
            ntm = ld_spinor(inj, sb + itm);
            if (edge)
                nh = ld_spinor(inj, sb + ie);
        }
        Spinor<R> vxp{shfl_c(cur.s0, lp), shfl_c(cur.s1, lp)};
        Spinor<R> vxm{shfl_c(cur.s0, lm), shfl_c(cur.s1, lm)};
        if (lane == 31)
            vxp = h;
        if (lane == 0)
            vxm = h;
        T up, lo;
        hop4<DAG, R>(vtp, vtm, vxp, vxm, Ut, Utm, Ux, Uxm, stp, stm, sxp, sxm, up, lo);
        Spinor<R> o{dg * cur.s0 - R(0.5) * up, dg * cur.s1 - R(0.5) * lo};
        if (L.fifth)
        {
            // D: spin 1 from s+1 (m_f psi(0) at the top), spin 0 from s-1 (m_f psi(Ls-1)
            // at 0); D^dag: the directions swapped
            const R cup = (s + 1 == Ls) ? mf : R(-1);
            const R cdn = (s == 0) ? mf : R(-1);
            if (!DAG)
            {
                o.s1 += cup * nxt.s1;
                o.s0 += cdn * prev.s0;
            }
            else
            {
                o.s1 += cdn * prev.s1;
                o.s0 += cup * nxt.s0;
            }
        }
        st_spinor(outj, long(s) * V + here, o);
        prev = cur;
        cur = nxt;
        vtp = ntp;
        vtm = ntm;
        h = nh;
    }
}

#define DWFB_COLX(DAG, R)                                                                         \
    template __global__ void dirac_colx_kernel<DAG, R>(Lat, const cplx<R>*, cplx<R>*, long,       \
                                                       const cplx<R>*, long, const int*, int);
DWFB_COLX(false, double)
DWFB_COLX(true, double)
DWFB_COLX(false, float)
DWFB_COLX(true, float)
#undef DWFB_COLX

// ---------------------------------------------------------------------------
// Column kernel over a block-shared slice ring filled by bulk copies
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tile_mbar_init(uint32_t mb, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mb), "r"(count));
}

__device__ __forceinline__ void tile_expect_tx(uint32_t mb, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> this CTA's shared memory, completing on mbarrier mb
// (both addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void tile_bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mb)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(mb)
        : "memory");
}

// Wait for the phase of parity `par` of mbarrier mb; false once limit_ns has
// passed (the timer is read every 64 polls).
__device__ __forceinline__ bool tile_wait(uint32_t mb, uint32_t par, unsigned long long limit_ns)
{
    unsigned long long t0 = 0;
    for (int it = 0;; ++it)
    {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mb), "r"(par)
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

template <bool DAG, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? DWFB_TILE_MINB64 : DWFB_TILE_MINB32)
    dirac_tile_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out, long fsz,
                      const cplx<R>* __restrict__ U, long usz, const int* __restrict__ conf,
                      int conf0, int* err, unsigned long long limit_ns)
{
    using T = cplx<R>;
    constexpr int NS = kRingSlots, NW = kRingT;
    constexpr uint32_t SB = 2 * sizeof(T);           // bytes of one site's spinor
    constexpr int kSlot = kRingRows * kRingWidth;    // sites per ring slot
    constexpr int kPrev = DAG ? 1 : 0, kNext = DAG ? 0 : 1;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    const T* ring = reinterpret_cast<const T*>(tile_smem);
    const uint32_t ring0 = uint32_t(__cvta_generic_to_shared(tile_smem));
    // after the ring: full[k][w] (warp w's rows of slot k landed), empty[k]
    // (all warps done with slot k)
    const uint32_t full0 = ring0 + NS * kSlot * SB;
    const uint32_t empty0 = full0 + 8 * NS * NW;

    const int j = blockIdx.z;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int Nt = L.Nt, Nx = L.Nx, V = L.V, Ls = L.Ls;
    const int x0 = blockIdx.x * 32, t0 = blockIdx.y * NW;
    const int t = t0 + warp, x = x0 + lane;
    const int c = conf ? conf[j] : conf0;
    const T* __restrict__ Uj = U + long(c) * usz;
    const T* __restrict__ inj = in + j * fsz;
    T* __restrict__ outj = out + j * fsz;

    if (threadIdx.x == 0)
    {
        for (int k = 0; k < NS * NW; ++k)
            tile_mbar_init(full0 + 8 * k, 1);
        for (int k = 0; k < NS; ++k)
            tile_mbar_init(empty0 + 8 * k, NW);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // Warp w copies ring row w + 1 (its own t row) of each slice, warp 0 also
    // row 0 (t0 - 1) and warp NW - 1 row NW + 1 (t0 + NW): per row, lane 3i
    // the sites x0 - 1 .. x0 + 32 that do not cross the x boundary, lanes
    // 3i + 1 and 3i + 2 the one site on either side that does (periodic in t and x).
    const int row_a = (warp == 0) ? 0 : warp + 1;
    const int nrows = (warp == 0 || warp == NW - 1) ? 2 : 1;
    auto issue = [&](int s) {
        const int k = s % NS;
        const uint32_t mb = full0 + 8 * (k * NW + warp);
        if (lane == 0)
            tile_expect_tx(mb, uint32_t(nrows * kRingWidth) * SB);
        __syncwarp();
        if (lane < 3 * nrows)
        {
            const int r = row_a + lane / 3, part = lane % 3;
            int tr = t0 - 1 + r;
            tr = tr < 0 ? tr + Nt : (tr >= Nt ? tr - Nt : tr);
            const T* row = inj + 2 * (long(s) * V + long(tr) * Nx);
            const uint32_t dst = ring0 + uint32_t(k * kSlot + r * kRingWidth) * SB;
            const int lo = (x0 == 0) ? 1 : 0, hi = (x0 + 32 == Nx) ? kRingWidth - 1 : kRingWidth;
            if (part == 0)
                tile_bulk_g2s(dst + lo * SB, row + 2 * (x0 - 1 + lo), uint32_t(hi - lo) * SB, mb);
            else if (part == 1 && lo)
                tile_bulk_g2s(dst, row + 2 * (Nx - 1), SB, mb);
            else if (part == 2 && hi < kRingWidth)
                tile_bulk_g2s(dst + (kRingWidth - 1) * SB, row, SB, mb);
        }
    };
    for (int s = 0; s < NS && s < Ls; ++s)
        issue(s);
    int issued = NS < Ls ? NS : Ls;  // slices 0 .. issued - 1 copied or in flight

    // link phases with the boundary signs folded in
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const int here = t * Nx + x;
    const T Ut = ((t == Nt - 1) ? R(L.bct) : R(1)) * Uj[here];
    const T Utm = ((t == 0) ? R(L.bct) : R(1)) * Uj[tm * Nx + x];
    const T Ux = ((x == Nx - 1) ? R(L.bcx) : R(1)) * Uj[V + here];
    const T Uxm = ((x == 0) ? R(L.bcx) : R(1)) * Uj[V + t * Nx + xm];
    const R dg = R(L.diag), mf = R(L.mf);
    T pv = {}, first_c = {};
    if (L.fifth)
        pv = inj[2 * (long(Ls - 1) * V + here) + kPrev];
    const int rc = (warp + 1) * kRingWidth + lane + 1;  // this site in a slot
    // the warps whose rows this warp reads: rows warp .. warp + 2 of a slot
    const int w_lo = warp > 0 ? warp - 1 : 0, w_hi = warp < NW - 1 ? warp + 1 : NW - 1;

    int s = 0;
    for (; s < Ls; ++s)
    {
        const int k = s % NS;
        const uint32_t par = (s / NS) & 1;
        bool ok = tile_wait(full0 + 8 * (k * NW + w_lo), par, limit_ns) &&
                  tile_wait(full0 + 8 * (k * NW + warp), par, limit_ns) &&
                  tile_wait(full0 + 8 * (k * NW + w_hi), par, limit_ns);
        if (ok && L.fifth && s + 1 < Ls)
            ok = tile_wait(full0 + 8 * (((s + 1) % NS) * NW + warp), ((s + 1) / NS) & 1, limit_ns);
        if (!__all_sync(0xffffffffu, ok))
            break;
        const T* S = ring + 2 * k * kSlot;
        const Spinor<R> cur = ld_spinor(S, rc);
        const Spinor<R> vtp = ld_spinor(S, rc + kRingWidth);
        const Spinor<R> vtm = ld_spinor(S, rc - kRingWidth);
        const Spinor<R> vxp = ld_spinor(S, rc + 1);
        const Spinor<R> vxm = ld_spinor(S, rc - 1);
        T up, lo;
        hop4<DAG, R>(vtp, vtm, vxp, vxm, Ut, Utm, Ux, Uxm, R(1), R(1), R(1), R(1), up, lo);
        Spinor<R> o{dg * cur.s0 - R(0.5) * up, dg * cur.s1 - R(0.5) * lo};
        if (L.fifth)
        {
            if (s == 0)
                first_c = kNext ? cur.s1 : cur.s0;
            const R cup = (s + 1 == Ls) ? mf : R(-1);
            const R cdn = (s == 0) ? mf : R(-1);
            const T nc = (s + 1 < Ls) ? ring[2 * (((s + 1) % NS) * kSlot + rc) + kNext] : first_c;
            if (!DAG)
            {
                o.s1 += cup * nc;
                o.s0 += cdn * pv;
            }
            else
            {
                o.s1 += cdn * pv;
                o.s0 += cup * nc;
            }
            pv = kPrev ? cur.s1 : cur.s0;
        }
        st_spinor(outj, long(s) * V + here, o);
        // this warp is done with slot k (its slice s + 1 component was read at step s)
        __syncwarp();
        if (lane == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(empty0 + 8 * k) : "memory");
        // refill the slot freed at the previous step once every warp is done with it
        if (s >= 1 && issued < Ls)
        {
            const int q = s - 1;
            const bool free = tile_wait(empty0 + 8 * (q % NS), (q / NS) & 1, limit_ns);
            if (!__all_sync(0xffffffffu, free))
                break;
            issue(issued);
            ++issued;
        }
    }
    if (s < Ls)
    {
        // a wait ran out: record it, and let this warp's copies in flight
        // (slices s .. issued - 1) land before it exits (allowing them at
        // least a second, however short the caller's limit)
        if (lane == 0)
        {
            atomicCAS(err, 0, int(DWF_TIMEOUT));
            const unsigned long long drain = limit_ns > 1000000000ull ? limit_ns : 1000000000ull;
            for (int q = s; q < issued; ++q)
                tile_wait(full0 + 8 * ((q % NS) * NW + warp), (q / NS) & 1, drain);
        }
    }
}

#define DWFB_TILE(DAG, R)                                                                          \
    template __global__ void dirac_tile_kernel<DAG, R>(Lat, const cplx<R>*, cplx<R>*, long,         \
                                                       const cplx<R>*, long, const int*, int, int*, \
                                                       unsigned long long);
DWFB_TILE(false, double)
DWFB_TILE(true, double)
DWFB_TILE(false, float)
DWFB_TILE(true, float)
#undef DWFB_TILE

template __global__ void dirac_col_kernel<false, double>(Lat, const double2*, double2*, long,
                                                         const double2*, long, const int*, int);
template __global__ void dirac_col_kernel<true, double>(Lat, const double2*, double2*, long,
                                                        const double2*, long, const int*, int);
template __global__ void dirac_col_kernel<false, float>(Lat, const float2*, float2*, long,
                                                        const float2*, long, const int*, int);
template __global__ void dirac_col_kernel<true, float>(Lat, const float2*, float2*, long,
                                                       const float2*, long, const int*, int);

namespace {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Ring-slot spinor storage. FP64: two planes (spin 0, spin 1) of Ls x W
// complex numbers, so that each 16-byte shared load of a warp is contiguous;
// FP32: one array of 16-byte spinors. `plane` = Ls * W; `off` = s * W + column.
__device__ __forceinline__ void cp_slot_spinor(double2* sl, int off, int plane, const double2* g)
{
    cp_async16(sl + off, g);
    cp_async16(sl + plane + off, g + 1);
}
__device__ __forceinline__ void cp_slot_spinor(float2* sl, int off, int, const float2* g)
{
    cp_async16(sl + 2 * off, g);
}
__device__ __forceinline__ Spinor<double> ld_slot_spinor(const double2* sl, int off, int plane)
{
    return {sl[off], sl[plane + off]};
}
__device__ __forceinline__ Spinor<float> ld_slot_spinor(const float2* sl, int off, int)
{
    const float4 v = reinterpret_cast<const float4*>(sl)[off];
    return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ double2 ld_slot_s0(const double2* sl, int off, int) { return sl[off]; }
__device__ __forceinline__ double2 ld_slot_s1(const double2* sl, int off, int plane)
{
    return sl[plane + off];
}
__device__ __forceinline__ float2 ld_slot_s0(const float2* sl, int off, int) { return sl[2 * off]; }
__device__ __forceinline__ float2 ld_slot_s1(const float2* sl, int off, int) { return sl[2 * off + 1]; }
__device__ __forceinline__ void cp_link(double2* d, const double2* g) { cp_async16(d, g); }
__device__ __forceinline__ void cp_link(float2* d, const float2* g) { cp_async8(d, g); }

}  // namespace

// o + a w and o + a (i w), one fused multiply-add per component
template <typename T, typename R>
__device__ __forceinline__ T caxpy(R a, T w, T o)
{
    return mkc(fma(a, w.x, o.x), fma(a, w.y, o.y));
}
template <typename T, typename R>
__device__ __forceinline__ T caxpy_i(R a, T w, T o)
{
    return mkc(fma(-a, w.y, o.x), fma(a, w.x, o.y));
}

// One block per (t chunk, G tiles of 32 consecutive x, all Ls slices), one
// thread per (s, x). The block streams the rows t0-1 .. t1 of its tile
// through a ring of (NPG + 1) * RPS shared-memory row slots with cp.async, in
// groups of RPS rows (NPG - 1 groups in flight while RPS rows are computed;
// no registers held for them): a slot holds the row's spinors for every s
// with one halo column on each side, and its t and x links. Each step a
// thread computes RPS consecutive rows of its own (s, x) from a register
// window of rows t-1 .. t+RPS, with the x +- 1 and s +- 1 neighbours and the
// links read from the slot of the row; one barrier per step. Every input
// spinor is loaded once per chunk (plus the two halo rows and columns). The
// boundary signs and the -1/2 of the hopping term are folded into the
// accumulation coefficients (one fused multiply-add per component and hop).
template <bool DAG, typename R, int NPG, int RPS>
__global__ void __launch_bounds__(512, (sizeof(R) == 8 && RPS == 2) ? 1 : 2)
    dirac_sweep_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                       long fsz, const cplx<R>* __restrict__ U, long usz,
                       const int* __restrict__ conf, int conf0, int tc)
{
    static_assert(RPS >= 1 && RPS <= 2, "one or two rows per step");
    // rows needed by step q end in group q + A; the pending-group count must be >= 0
    constexpr int A = (RPS + 1) / RPS;
    static_assert(NPG - 1 - A >= 0, "prologue too short for the rows a step needs");
    constexpr int NS = (NPG + 1) * RPS;                  // row slots in the ring
    using T = cplx<R>;
    extern __shared__ __align__(16) unsigned char sweep_smem[];
    const int j = blockIdx.z;
    const int c = conf ? conf[j] : conf0;
    const T* __restrict__ Uj = U + long(c) * usz;
    const int lane = threadIdx.x, s = threadIdx.y, g = threadIdx.z, G = blockDim.z;
    const int Nt = L.Nt, Nx = L.Nx, V = L.V, Ls = L.Ls;
    const int xb = blockIdx.x * G * 32;                  // first x of the block
    const int x = xb + g * 32 + lane;
    const int xl = (xb == 0) ? Nx - 1 : xb - 1;          // left halo column
    const int xr = (xb + 32 * G == Nx) ? 0 : xb + 32 * G; // right halo column
    const int t0 = blockIdx.y * tc;
    const int t1 = min(t0 + tc, Nt);
    const int nrow = t1 - t0 + 2;                        // rows t0-1 .. t1
    const int W = 32 * G + 2;                            // slot row width (with halos)
    const int i = g * 32 + lane + 1;                     // this thread's column in a slot
    const int plane = Ls * W;
    const int own = s * W + i;
    const int sup = (s + 1 == Ls) ? 0 : s + 1;
    const int sdn = (s == 0) ? Ls - 1 : s - 1;
    // fifth-dimension sources of spin 1 and spin 0 (D: s+1 and s-1; D^dag: swapped)
    const int off_s1 = (DAG ? sdn : sup) * W + i;
    const int off_s0 = (DAG ? sup : sdn) * W + i;
    const int slot_c = int(sweep_slot_bytes(Ls, G, sizeof(T)) / sizeof(T));  // complex per slot
    const int ring_c = NS * slot_c;
    T* const ring = reinterpret_cast<T*>(sweep_smem);
    const int lt = 2 * plane + i - 1;                    // t link of this column
    const int lx = 2 * plane + 32 * G + i;               // x link; lx - 1 is the one at x - 1

    const bool halo_l = (g == 0 && lane == 0), halo_r = (g == G - 1 && lane == 31);
    const bool extra = halo_l || halo_r || s == 0;      // copies more than its own spinor
    const long rstride = 2L * Nx;                        // complex numbers per row

    // Fetch state: the next chunk row (ri, at t = ti) with running pointers to
    // this thread's spinor and links in that row; halo columns are fixed
    // offsets from them.
    int ri = 0;
    int ti = (t0 == 0) ? Nt - 1 : t0 - 1;
    const T* gp = in + j * fsz + 2 * (long(s) * V + long(ti) * Nx + x);
    const T* up = Uj + ti * Nx + x;                      // t link; the x link is up + V
    const long hl = 2L * (xl - x), hr = 2L * (xr - x);
    const int ul = xl - x;
    int bf = 0;                                          // slot (complex offset) of the next row

    auto fetch_row = [&]() {
        if (ri < nrow)
        {
            T* const d = ring + bf;
            cp_slot_spinor(d, own, plane, gp);
            if (extra)
            {
                if (halo_l)
                    cp_slot_spinor(d, own - 1, plane, gp + hl);
                if (halo_r)
                    cp_slot_spinor(d, own + 1, plane, gp + hr);
                if (s == 0)
                {
                    cp_link(d + lt, up);
                    cp_link(d + lx, up + V);
                    if (halo_l)
                        cp_link(d + lx - 1, up + V + ul);
                }
            }
            ++ri;
            if (++ti == Nt)
            {
                ti = 0;
                gp -= (Nt - 1) * rstride;
                up -= (Nt - 1) * Nx;
            }
            else
            {
                gp += rstride;
                up += Nx;
            }
        }
        bf = (bf + slot_c == ring_c) ? 0 : bf + slot_c;
    };
    // one commit group of RPS rows, empty past the last row so that the
    // group count per step stays fixed
    auto fetch_group = [&]() {
        for (int d = 0; d < RPS; ++d)
            fetch_row();
        cp_async_commit();
    };

    const R half = R(0.5);
    const R cbt = -half * R(L.bct);                      // -1/2 times the t boundary sign
    constexpr R kf = DAG ? R(1) : R(-1);
    constexpr R kb = -kf;
    const R cxp = (x == Nx - 1) ? -half * R(L.bcx) : -half;
    const R cxm = (x == 0) ? -half * R(L.bcx) : -half;
    const R dg = R(L.diag);
    // D: spin 1 from s+1 (m_f psi(0) at the top), spin 0 from s-1 (m_f psi(Ls-1) at 0);
    // D^dag: the directions swapped.
    const R c5_1 = DAG ? ((s == 0) ? R(L.mf) : R(-1)) : ((s + 1 == Ls) ? R(L.mf) : R(-1));
    const R c5_0 = DAG ? ((s + 1 == Ls) ? R(L.mf) : R(-1)) : ((s == 0) ? R(L.mf) : R(-1));
    T* __restrict__ op = out + j * fsz + 2 * (long(s) * V + long(t0) * Nx + x);

    // output of row t from its slot pc, the rows t-1, t, t+1 of this column and
    // the backward t link
    auto site = [&](const T* pc, const Spinor<R>& pv, const Spinor<R>& cu, const Spinor<R>& nx,
                    const T& Utm, int t) {
        const Spinor<R> vxp = ld_slot_spinor(pc, own + 1, plane);
        const Spinor<R> vxm = ld_slot_spinor(pc, own - 1, plane);
        const T Ut = pc[lt];
        const T Ux = pc[lx];
        const T Uxm = pc[lx - 1];
        const R ctp = (t == Nt - 1) ? cbt : -half;
        const R ctm = (t == 0) ? cbt : -half;
        Spinor<R> o{dg * cu.s0, dg * cu.s1};
        T w = cmul(Ut, nx.s0 + kf * nx.s1);
        o.s0 = caxpy(ctp, w, o.s0);
        o.s1 = caxpy(kf * ctp, w, o.s1);
        w = cmulc(Utm, pv.s0 + kb * pv.s1);
        o.s0 = caxpy(ctm, w, o.s0);
        o.s1 = caxpy(kb * ctm, w, o.s1);
        w = cmul(Ux, vxp.s0 - kf * itimes(vxp.s1));
        o.s0 = caxpy(cxp, w, o.s0);
        o.s1 = caxpy_i(kf * cxp, w, o.s1);
        w = cmulc(Uxm, vxm.s0 - kb * itimes(vxm.s1));
        o.s0 = caxpy(cxm, w, o.s0);
        o.s1 = caxpy_i(kb * cxm, w, o.s1);
        if (L.fifth)
        {
            o.s1 = caxpy(c5_1, ld_slot_s1(pc, off_s1, plane), o.s1);
            o.s0 = caxpy(c5_0, ld_slot_s0(pc, off_s0, plane), o.s0);
        }
        return o;
    };
    auto slot_at = [&](int b, int d) {   // slot d rows after slot b
        const int o = b + d * slot_c;
        return (o >= ring_c) ? o - ring_c : o;
    };

    for (int q = 0; q < NPG; ++q)
        fetch_group();
    // b0: slot of row t-1 for the first output row t of the step
    int b0 = 0;
    Spinor<R> prev = {}, cur = {};
    T Utm = {};
    for (int t = t0; t < t1; t += RPS)
    {
        // the rows t-1 .. t+RPS are complete for every thread
        cp_async_wait<NPG - 1 - A>();
        __syncthreads();
        fetch_group();   // into the slots of the previous step's first rows
        const T* const p1 = ring + slot_at(b0, 1);
        if (t == t0)
        {
            prev = ld_slot_spinor(ring, own, plane);
            cur = ld_slot_spinor(p1, own, plane);
            Utm = ring[lt];
        }
        const Spinor<R> n1 = ld_slot_spinor(ring + slot_at(b0, 2), own, plane);
        st_spinor(op, 0, site(p1, prev, cur, n1, Utm, t));
        op += rstride;
        if (RPS == 2)
        {
            const T Ut = p1[lt];
            if (t + 1 < t1)
            {
                const T* const p2 = ring + slot_at(b0, 2);
                const Spinor<R> n2 = ld_slot_spinor(ring + slot_at(b0, 3), own, plane);
                st_spinor(op, 0, site(p2, cur, n1, n2, Ut, t + 1));
                op += rstride;
                Utm = p2[lt];
                prev = n1;
                cur = n2;
            }
        }
        else
        {
            Utm = p1[lt];
            prev = cur;
            cur = n1;
        }
        b0 = slot_at(b0, RPS);
    }
    cp_async_wait<0>();
}

#define DWFB_SWEEP_INST(DAG, R, NPG, RPS)                                                         \
    template __global__ void dirac_sweep_kernel<DAG, R, NPG, RPS>(                                \
        Lat, const cplx<R>*, cplx<R>*, long, const cplx<R>*, long, const int*, int, int);
DWFB_SWEEP_INST(false, double, kSweepGroups64, kSweepRows64)
DWFB_SWEEP_INST(true, double, kSweepGroups64, kSweepRows64)
DWFB_SWEEP_INST(false, float, kSweepGroups32, kSweepRows32)
DWFB_SWEEP_INST(true, float, kSweepGroups32, kSweepRows32)
#undef DWFB_SWEEP_INST

template __global__ void dirac_kernel<false, double>(Lat, const double2*, double2*, long,
                                                     const double2*, long, const int*, int);
template __global__ void dirac_kernel<true, double>(Lat, const double2*, double2*, long,
                                                    const double2*, long, const int*, int);
template __global__ void dirac_kernel<false, float>(Lat, const float2*, float2*, long,
                                                    const float2*, long, const int*, int);
template __global__ void dirac_kernel<true, float>(Lat, const float2*, float2*, long,
                                                   const float2*, long, const int*, int);

template <bool DAG>
__global__ void __launch_bounds__(256)
    residual_partials_kernel(Lat L, const double2* __restrict__ t, const double2* __restrict__ b,
                             long fsz, const double2* __restrict__ U, long usz,
                             const int* __restrict__ conf, int nch, int ch,
                             double* __restrict__ part)
{
    __shared__ double scratch[64];
    const int j = blockIdx.y, c = blockIdx.x;
    const double2* Uj = U + long(conf[j]) * usz;
    const int beg = c * ch, end = min(beg + ch, L.nsite);
    double rr = 0.0, bb = 0.0;
    for (int i = beg + threadIdx.x; i < end; i += blockDim.x)
    {
        int s, tt, x;
        site_coords(L, i, s, tt, x);
        const Spinor<double> a = dirac_site<DAG, double>(t + j * fsz, Uj, L, s, tt, x);
        const Spinor<double> bv = ld_spinor(b + j * fsz, i);
        const Spinor<double> r = {bv.s0 - a.s0, bv.s1 - a.s1};
        rr += spinor_norm2(r);
        bb += spinor_norm2(bv);
    }
    rr = block_sum(rr, scratch);
    bb = block_sum(bb, scratch);
    if (threadIdx.x == 0)
    {
        part[(long(j) * nch + c) * 2] = rr;
        part[(long(j) * nch + c) * 2 + 1] = bb;
    }
}

template __global__ void residual_partials_kernel<false>(Lat, const double2*, const double2*,
                                                         long, const double2*, long, const int*,
                                                         int, int, double*);
template __global__ void residual_partials_kernel<true>(Lat, const double2*, const double2*, long,
                                                        const double2*, long, const int*, int,
                                                        int, double*);

__global__ void residual_finish_kernel(const double* __restrict__ part, int nrhs, int nch,
                                       double* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (j >= nrhs)
        return;
    double rr = 0.0, bb = 0.0;
    for (int c = lane; c < nch; c += 32)
    {
        rr += part[(long(j) * nch + c) * 2];
        bb += part[(long(j) * nch + c) * 2 + 1];
    }
    rr = warp_sum(rr);
    bb = warp_sum(bb);
    if (lane == 0)
        out[j] = bb > 0.0 ? sqrt(rr / bb) : 0.0;
}

// Every block passes `rounds` grid barriers that expect `expected` arrivals.
// With expected > gridDim.x no barrier can complete: each wait runs into its
// limit and records DWF_TIMEOUT, and every block returns.
__global__ void barrier_probe_kernel(GridBar* bar, unsigned expected, unsigned long long timeout_ns,
                                     int rounds)
{
    for (int k = 0; k < rounds; ++k)
        if (!grid_sync(bar, expected, timeout_ns))
            return;
}

}  // namespace dwfb
