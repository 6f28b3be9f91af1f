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
