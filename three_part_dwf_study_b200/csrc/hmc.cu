// HMC on the device: gauge and pseudofermion forces, leapfrog kick/drift and
// the trajectory orchestration for both formulations.
#include <algorithm>
#include <cmath>
#include <vector>

#include "context.cuh"
#include "hmc.cuh"
#include "kernels.cuh"

namespace dwfb {

__device__ __forceinline__ double plaq_angle(const double* th, int Nt, int Nx, int t, int x)
{
    const int tp = (t + 1 == Nt) ? 0 : t + 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int V = Nt * Nx;
    return th[t * Nx + x] + th[V + tp * Nx + x] - th[t * Nx + xp] - th[V + t * Nx + x];
}

__global__ void __launch_bounds__(256)
    gauge_force_kernel(int Nt, int Nx, double beta, const double* __restrict__ th,
                       double* __restrict__ force, double* __restrict__ part)
{
    __shared__ double scratch[64];
    const int V = Nt * Nx;
    double act = 0.0, cs = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x)
    {
        const int t = i / Nx, x = i - t * Nx;
        const int tm = (t == 0) ? Nt - 1 : t - 1;
        const int xm = (x == 0) ? Nx - 1 : x - 1;
        const double p = plaq_angle(th, Nt, Nx, t, x);
        const double here = sin(p);
        // F_t(t,x) = beta (sin P(t,x) - sin P(t,x-1)); F_x(t,x) = beta (sin P(t-1,x) - sin P(t,x))
        force[i] = beta * (here - sin(plaq_angle(th, Nt, Nx, t, xm)));
        force[V + i] = beta * (sin(plaq_angle(th, Nt, Nx, tm, x)) - here);
        const double c = cos(p);
        act += beta * (1.0 - c);
        cs += c;
    }
    act = block_sum(act, scratch);
    cs = block_sum(cs, scratch);
    if (threadIdx.x == 0)
    {
        part[2 * blockIdx.x] = act;
        part[2 * blockIdx.x + 1] = cs;
    }
}

// For link (mu, y) with neighbour n = y + mu:
//   A = sum_s eta(s,y)^dag (1 - gamma_mu) xi(s,n),  B = sum_s eta(s,n)^dag (1 + gamma_mu) xi(s,y)
//   F = -bc Im(U A - U^* B)
// which is -2 Re[(-i/2) bc U A + (i/2) bc U^* B], the forward term of site y
// plus the backward term of site n shifted onto the link (the reference's
// "np.roll" step, pseudofermion.hpp:139-157; wilson/include/gauge.hpp:110-118).
// Projected forms: eta^dag (1 + k gamma) xi = conj(eta0 + k g^* eta1) (xi0 + k g^* xi1)
// with g = 1 for gamma_t = sigma1 and g = i for gamma_x = sigma2.
__global__ void __launch_bounds__(256)
    pf_force_kernel(Lat L, const double2* __restrict__ eta, const double2* __restrict__ xi,
                    const double2* __restrict__ U, double* __restrict__ force)
{
    const int V = L.V;
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < 2 * V; l += gridDim.x * blockDim.x)
    {
        const int mu = l / V, y = l - mu * V;
        const int t = y / L.Nx, x = y - t * L.Nx;
        int n;
        double bc;
        if (mu == 0)
        {
            n = ((t + 1 == L.Nt) ? 0 : t + 1) * L.Nx + x;
            bc = (t == L.Nt - 1) ? L.bct : 1.0;
        }
        else
        {
            n = t * L.Nx + ((x + 1 == L.Nx) ? 0 : x + 1);
            bc = (x == L.Nx - 1) ? L.bcx : 1.0;
        }
        double2 A = make_double2(0.0, 0.0), B = make_double2(0.0, 0.0);
        for (int s = 0; s < L.Ls; ++s)
        {
            const long sb = long(s) * V;
            const Spinor<double> ey = ld_spinor(eta, sb + y);
            const Spinor<double> en = ld_spinor(eta, sb + n);
            const Spinor<double> xy = ld_spinor(xi, sb + y);
            const Spinor<double> xn = ld_spinor(xi, sb + n);
            if (mu == 0)
            {
                A += cmulc(ey.s0 - ey.s1, xn.s0 - xn.s1);  // (1 - sigma1)
                B += cmulc(en.s0 + en.s1, xy.s0 + xy.s1);  // (1 + sigma1)
            }
            else
            {
                A += cmulc(ey.s0 + itimes(ey.s1), xn.s0 + itimes(xn.s1));  // (1 - sigma2)
                B += cmulc(en.s0 - itimes(en.s1), xy.s0 - itimes(xy.s1));  // (1 + sigma2)
            }
        }
        const double2 u = U[l];
        const double2 ua = cmul(u, A);
        const double2 ub = cmulc(u, B);
        force[l] += -bc * (ua.y - ub.y);
    }
}

__global__ void __launch_bounds__(256)
    dot_re_kernel(const double2* __restrict__ a, const double2* __restrict__ b, long n,
                  double* __restrict__ part)
{
    __shared__ double scratch[64];
    double s = 0.0;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n;
         i += long(gridDim.x) * blockDim.x)
        s += a[i].x * b[i].x + a[i].y * b[i].y;
    s = block_sum(s, scratch);
    if (threadIdx.x == 0)
        part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256)
    kinetic_kernel(const double* __restrict__ p, long n, double* __restrict__ part)
{
    __shared__ double scratch[64];
    double s = 0.0;
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n;
         i += long(gridDim.x) * blockDim.x)
        s += 0.5 * p[i] * p[i];
    s = block_sum(s, scratch);
    if (threadIdx.x == 0)
        part[blockIdx.x] = s;
}

__global__ void finish_sum_kernel(const double* __restrict__ part, int nblk, int stride,
                                  double* __restrict__ out)
{
    __shared__ double scratch[64];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        s += part[b * stride];
    s = block_sum(s, scratch);
    if (threadIdx.x == 0)
        out[0] = s;
}

__global__ void kick_kernel(double* __restrict__ mom, const double* __restrict__ force, double c,
                            long n)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n;
         i += long(gridDim.x) * blockDim.x)
        mom[i] -= c * force[i];
}

// wrap_angle (wilson/include/indexing.hpp:13-18): fmod is exact, so the
// wrapped angle is bit-identical to the host computation.
__device__ __forceinline__ double wrap_angle(double a)
{
    const double pi = 3.14159265358979323846;
    a = fmod(a + pi, 2.0 * pi);
    if (a < 0.0)
        a += 2.0 * pi;
    return a - pi;
}

__global__ void drift_kernel(double* __restrict__ th, const double* __restrict__ mom, double eps,
                             int wrap, long n, double2* __restrict__ U64, float2* __restrict__ U32)
{
    for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n;
         i += long(gridDim.x) * blockDim.x)
    {
        double v = th[i] + eps * mom[i];
        if (wrap)
            v = wrap_angle(v);
        th[i] = v;
        double sn, cs;
        sincos(v, &sn, &cs);
        U64[i] = make_double2(cs, sn);
        U32[i] = make_float2(float(cs), float(sn));
    }
}

}  // namespace dwfb
