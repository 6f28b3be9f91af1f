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

// One block per (t chunk, G tiles of 32 consecutive x, all Ls slices), one
// thread per (s, x). The block streams the rows t0-1 .. t1 of its tile
// through a ring of S shared-memory slots with cp.async (S-3 rows in flight
// while a row is computed; no registers held for them): a slot holds the
// row's spinors for every s with one halo column on each side, and its t and
// x links. Each thread keeps its own rows t-1, t, t+1 in registers and reads
// the x +- 1 and s +- 1 neighbours and the links from the slot of row t. One
// barrier per row. Every input spinor is loaded once per chunk (plus the two
// halo rows and the two halo columns).
template <bool DAG, typename R, int S>
__global__ void __launch_bounds__(512, 2)
    dirac_sweep_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                       long fsz, const cplx<R>* __restrict__ U, long usz,
                       const int* __restrict__ conf, int conf0, int tc)
{
    static_assert(S >= 4, "the ring holds rows t-1, t, t+1 and the slot being refilled");
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
    const int off_up = sup * W + i, off_dn = sdn * W + i;
    const int slot_c = int(sweep_slot_bytes(Ls, G, sizeof(T)) / sizeof(T));  // complex per slot
    T* const ring = reinterpret_cast<T*>(sweep_smem);
    const int lk = 2 * plane;                            // links after the spinors

    // this thread's input column (s, x) at row 0, its halo columns
    const T* __restrict__ gin = in + j * fsz + 2 * (long(s) * V + x);
    const T* __restrict__ gxl = in + j * fsz + 2 * (long(s) * V + xl);
    const T* __restrict__ gxr = in + j * fsz + 2 * (long(s) * V + xr);
    const bool halo_l = (g == 0 && lane == 0), halo_r = (g == G - 1 && lane == 31);
    const long rstride = 2L * Nx;                        // complex numbers per row

    // row r of the chunk (t = t0 - 1 + r, wrapped) into slot `sl`; one commit
    // group per row, empty past the last row so that the group count per step
    // stays fixed
    auto issue = [&](int r, int sl) {
        if (r < nrow)
        {
            int t = t0 - 1 + r;
            t = (t < 0) ? t + Nt : ((t >= Nt) ? t - Nt : t);
            T* const d = ring + sl * slot_c;
            const long ro = t * rstride;
            cp_slot_spinor(d, own, plane, gin + ro);
            if (halo_l)
                cp_slot_spinor(d, own - 1, plane, gxl + ro);
            if (halo_r)
                cp_slot_spinor(d, own + 1, plane, gxr + ro);
            if (s == 0)
            {
                cp_link(d + lk + i - 1, Uj + t * Nx + x);
                cp_link(d + lk + 32 * G + i, Uj + V + t * Nx + x);
                if (halo_l)
                    cp_link(d + lk + 32 * G, Uj + V + t * Nx + xl);
            }
        }
        cp_async_commit();
    };

    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    constexpr R kf = DAG ? R(1) : R(-1);
    constexpr R kb = -kf;
    const R dg = R(L.diag);
    const R cup = (s + 1 == Ls) ? R(L.mf) : R(-1);
    const R cdn = (s == 0) ? R(L.mf) : R(-1);
    T* __restrict__ ocol = out + j * fsz + 2 * (long(s) * V + x);

    for (int r = 0; r < S - 1; ++r)
        issue(r, r);
    // slots of rows k+1 (t), k+2 (t+1) and of the row being refilled (k-1)
    int sc = 1, sn = 2, sf = S - 1;
    Spinor<R> prev = {}, cur = {};
    T Utm = {};
    for (int k = 0; t0 + k < t1; ++k)
    {
        // rows k, k+1, k+2 (t-1, t, t+1) complete for every thread
        cp_async_wait<S - 4>();
        __syncthreads();
        issue(k + S - 1, sf);   // the slot of row k-1, which no thread reads any more
        const int t = t0 + k;
        const T* const pc = ring + sc * slot_c;
        if (k == 0)
        {
            prev = ld_slot_spinor(ring, own, plane);
            cur = ld_slot_spinor(pc, own, plane);
            Utm = ring[lk + i - 1];
        }
        const Spinor<R> next = ld_slot_spinor(ring + sn * slot_c, own, plane);
        const Spinor<R> vxp = ld_slot_spinor(pc, own + 1, plane);
        const Spinor<R> vxm = ld_slot_spinor(pc, own - 1, plane);
        const T Ut = pc[lk + i - 1];
        const T Ux = pc[lk + 32 * G + i];
        const T Uxm = pc[lk + 32 * G + i - 1];
        const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
        const R stm = (t == 0) ? R(L.bct) : R(1);

        T w = cmul(Ut, stp * (next.s0 + kf * next.s1));
        T hu = w;
        T hl = kf * w;
        w = cmulc(Utm, stm * (prev.s0 + kb * prev.s1));
        hu += w;
        hl += kb * w;
        w = cmul(Ux, sxp * (vxp.s0 - kf * itimes(vxp.s1)));
        hu += w;
        hl += kf * itimes(w);
        w = cmulc(Uxm, sxm * (vxm.s0 - kb * itimes(vxm.s1)));
        hu += w;
        hl += kb * itimes(w);
        Spinor<R> o{dg * cur.s0 - R(0.5) * hu, dg * cur.s1 - R(0.5) * hl};
        if (L.fifth)
        {
            // D: spin 1 from s+1 (m_f psi(0) at the top), spin 0 from s-1 (m_f psi(Ls-1) at 0);
            // D^dag: the directions swapped.
            if (!DAG)
            {
                o.s1 += cup * ld_slot_s1(pc, off_up, plane);
                o.s0 += cdn * ld_slot_s0(pc, off_dn, plane);
            }
            else
            {
                o.s1 += cdn * ld_slot_s1(pc, off_dn, plane);
                o.s0 += cup * ld_slot_s0(pc, off_up, plane);
            }
        }
        st_spinor(ocol + t * rstride, 0, o);
        prev = cur;
        cur = next;
        Utm = Ut;
        sc = (sc + 1 == S) ? 0 : sc + 1;
        sn = (sn + 1 == S) ? 0 : sn + 1;
        sf = (sf + 1 == S) ? 0 : sf + 1;
    }
    cp_async_wait<0>();
}

#define DWFB_SWEEP_INST(DAG, R, S)                                                               \
    template __global__ void dirac_sweep_kernel<DAG, R, S>(Lat, const cplx<R>*, cplx<R>*, long, \
                                                           const cplx<R>*, long, const int*, int,  \
                                                           int);
DWFB_SWEEP_INST(false, double, kSweepSlots64)
DWFB_SWEEP_INST(true, double, kSweepSlots64)
DWFB_SWEEP_INST(false, float, kSweepSlots32)
DWFB_SWEEP_INST(true, float, kSweepSlots32)
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
