// Wilson and domain-wall Dirac operators at one lattice site.
//
// Both operators share the 4-D hopping term
//   (D psi)(y) = diag psi(y)
//              - 1/2 sum_mu [ bc U_mu(y)       (1 - gamma_mu) psi(y + mu)
//                           + bc U_mu(y - mu)^* (1 + gamma_mu) psi(y - mu) ]
// with gamma_t = sigma1, gamma_x = sigma2 (domain_wall/include/spin.hpp:5-19,
// wilson/include/wilson_operator.hpp:13-14). D^dag swaps (1 - gamma) and
// (1 + gamma). diag = 3 - M5 for domain wall (dwf_operator.hpp:17), 2 + m0 for
// Wilson (wilson_operator.hpp:35). Boundary signs: domain wall is
// antiperiodic in t and periodic in x (dwf_operator.hpp:29-30); Wilson takes
// them from wilson.time/space_boundary_sign (wilson_operator.hpp:38-54).
//
// Domain wall adds the fifth-dimension hop (dwf_operator.hpp:71-86 for D,
// :150-165 for D^dag):
//   D    : spin 1 gets -psi_1(s+1) (m_f psi_1(0) at s = Ls-1),
//          spin 0 gets -psi_0(s-1) (m_f psi_0(Ls-1) at s = 0)
//   D^dag: spin 1 gets -psi_1(s-1) (m_f psi_1(Ls-1) at s = 0),
//          spin 0 gets -psi_0(s+1) (m_f psi_0(0) at s = Ls-1)
//
// Each hop is evaluated on its projected half-spinor: with
// (1 + k gamma) v = (h, k g h) where h = v0 + k g^* v1 and g = 1 for
// sigma1, g = i for sigma2, one complex link product per hop suffices.
#pragma once

#include "common.cuh"

namespace dwfb {

// Field loaders: dirac_site reads its input through one of these, so the
// same stencil can read a stored field or a combination formed on the fly.
template <typename R>
struct FieldLd
{
    const cplx<R>* __restrict__ f;
    __device__ __forceinline__ Spinor<R> sp(long site) const { return ld_spinor(f, site); }
    __device__ __forceinline__ cplx<R> c(long idx) const { return f[idx]; }
};

// x + e with x in FP64 and e in FP32 (the mixed solver's reliable update).
struct SumLd
{
    const double2* __restrict__ x;
    const float2* __restrict__ e;
    __device__ __forceinline__ Spinor<double> sp(long site) const
    {
        const Spinor<double> a = ld_spinor(x, site);
        const Spinor<float> b = ld_spinor(e, site);
        return {mkc(a.s0.x + double(b.s0.x), a.s0.y + double(b.s0.y)),
                mkc(a.s1.x + double(b.s1.x), a.s1.y + double(b.s1.y))};
    }
    __device__ __forceinline__ double2 c(long idx) const
    {
        const double2 a = x[idx];
        const float2 b = e[idx];
        return mkc(a.x + double(b.x), a.y + double(b.y));
    }
};

// The 4-D hopping sum of one site from its four neighbours' spinors, the
// links and the boundary signs: D psi = diag psi - (up, lo) / 2 (plus the
// fifth-dimension hop for domain wall). Forward hops use (1 + kf gamma),
// backward hops (1 + kb gamma).
template <bool DAG, typename R>
__device__ __forceinline__ void hop4(const Spinor<R>& vtp, const Spinor<R>& vtm,
                                     const Spinor<R>& vxp, const Spinor<R>& vxm, cplx<R> Ut,
                                     cplx<R> Utm, cplx<R> Ux, cplx<R> Uxm, R stp, R stm, R sxp,
                                     R sxm, cplx<R>& up, cplx<R>& lo)
{
    constexpr R kf = DAG ? R(1) : R(-1);
    constexpr R kb = -kf;
    cplx<R> w = cmul(Ut, stp * (vtp.s0 + kf * vtp.s1));
    up = w;
    lo = kf * w;
    w = cmulc(Utm, stm * (vtm.s0 + kb * vtm.s1));
    up += w;
    lo += kb * w;
    w = cmul(Ux, sxp * (vxp.s0 - kf * itimes(vxp.s1)));
    up += w;
    lo += kf * itimes(w);
    w = cmulc(Uxm, sxm * (vxm.s0 - kb * itimes(vxm.s1)));
    up += w;
    lo += kb * itimes(w);
}

// Link phases are stored per configuration as U[mu][t][x] = (cos, sin).
template <bool DAG, typename R, typename Ld>
__device__ __forceinline__ Spinor<R> dirac_site_ld(const Ld& in, const cplx<R>* __restrict__ U,
                                                const Lat& L, int s, int t, int x)
{
    using T = cplx<R>;
    const int Nt = L.Nt, Nx = L.Nx;
    const int tp = (t + 1 == Nt) ? 0 : t + 1;
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const long sb = long(s) * L.V;
    const int here = t * Nx + x;

    const Spinor<R> c = in.sp(sb + here);
    const Spinor<R> vtp = in.sp(sb + tp * Nx + x);
    const Spinor<R> vtm = in.sp(sb + tm * Nx + x);
    const Spinor<R> vxp = in.sp(sb + t * Nx + xp);
    const Spinor<R> vxm = in.sp(sb + t * Nx + xm);
    const T Ut = U[here];
    const T Utm = U[tm * Nx + x];
    const T Ux = U[L.V + here];
    const T Uxm = U[L.V + t * Nx + xm];

    const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
    const R stm = (t == 0) ? R(L.bct) : R(1);
    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    T up, lo;
    hop4<DAG, R>(vtp, vtm, vxp, vxm, Ut, Utm, Ux, Uxm, stp, stm, sxp, sxm, up, lo);

    const R dg = R(L.diag);
    Spinor<R> o;
    o.s0 = dg * c.s0 - R(0.5) * up;
    o.s1 = dg * c.s1 - R(0.5) * lo;

    if (L.fifth)
    {
        const int Ls = L.Ls;
        const int sup = (s + 1 == Ls) ? 0 : s + 1;
        const R cup = (s + 1 == Ls) ? R(L.mf) : R(-1);
        const int sdn = (s == 0) ? Ls - 1 : s - 1;
        const R cdn = (s == 0) ? R(L.mf) : R(-1);
        if (!DAG)
        {
            o.s1 += cup * in.c(2 * (long(sup) * L.V + here) + 1);
            o.s0 += cdn * in.c(2 * (long(sdn) * L.V + here));
        }
        else
        {
            o.s1 += cdn * in.c(2 * (long(sdn) * L.V + here) + 1);
            o.s0 += cup * in.c(2 * (long(sup) * L.V + here));
        }
    }
    return o;
}

template <bool DAG, typename R>
__device__ __forceinline__ Spinor<R> dirac_site(const cplx<R>* __restrict__ in,
                                                const cplx<R>* __restrict__ U, const Lat& L,
                                                int s, int t, int x)
{
    return dirac_site_ld<DAG, R>(FieldLd<R>{in}, U, L, s, t, x);
}

// Shuffle of a complex number / spinor between lanes of a full warp.
__device__ __forceinline__ double2 shfl_c(double2 v, int src)
{
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ float2 shfl_c(float2 v, int src)
{
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// The operator at (s, t, x) for a warp whose 32 lanes hold x = x0 .. x0 + 31 of
// one row (Nx a multiple of 32): the x +- 1 neighbours and the backward x link
// come from the adjacent lanes by shuffle (lanes 0 and 31 load theirs), so a
// site issues 3 spinor loads for the 4-D hop instead of 5.
template <bool DAG, typename R>
__device__ __forceinline__ Spinor<R> dirac_site_warp(const cplx<R>* __restrict__ in,
                                                     const cplx<R>* __restrict__ U, const Lat& L,
                                                     int s, int t, int x, int lane)
{
    using T = cplx<R>;
    const int Nt = L.Nt, Nx = L.Nx;
    const int tp = (t + 1 == Nt) ? 0 : t + 1;
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const long sb = long(s) * L.V;
    const int here = t * Nx + x;

    const Spinor<R> c = ld_spinor(in, sb + here);
    const T Ux = U[L.V + here];
    // neighbours in x from the adjacent lanes (same row, consecutive x)
    const int up = (lane == 31) ? 31 : lane + 1, dn = (lane == 0) ? 0 : lane - 1;
    Spinor<R> vxp{shfl_c(c.s0, up), shfl_c(c.s1, up)};
    Spinor<R> vxm{shfl_c(c.s0, dn), shfl_c(c.s1, dn)};
    T Uxm = shfl_c(Ux, dn);
    if (lane == 31)
        vxp = ld_spinor(in, sb + t * Nx + xp);
    if (lane == 0)
    {
        vxm = ld_spinor(in, sb + t * Nx + xm);
        Uxm = U[L.V + t * Nx + xm];
    }
    const Spinor<R> vtp = ld_spinor(in, sb + tp * Nx + x);
    const Spinor<R> vtm = ld_spinor(in, sb + tm * Nx + x);
    const T Ut = U[here];
    const T Utm = U[tm * Nx + x];

    const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
    const R stm = (t == 0) ? R(L.bct) : R(1);
    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    T upv, lo;
    hop4<DAG, R>(vtp, vtm, vxp, vxm, Ut, Utm, Ux, Uxm, stp, stm, sxp, sxm, upv, lo);

    const R dg = R(L.diag);
    Spinor<R> o;
    o.s0 = dg * c.s0 - R(0.5) * upv;
    o.s1 = dg * c.s1 - R(0.5) * lo;
    if (L.fifth)
    {
        const int Ls = L.Ls;
        const int sup = (s + 1 == Ls) ? 0 : s + 1;
        const R cup = (s + 1 == Ls) ? R(L.mf) : R(-1);
        const int sdn = (s == 0) ? Ls - 1 : s - 1;
        const R cdn = (s == 0) ? R(L.mf) : R(-1);
        if (!DAG)
        {
            o.s1 += cup * in[2 * (long(sup) * L.V + here) + 1];
            o.s0 += cdn * in[2 * (long(sdn) * L.V + here)];
        }
        else
        {
            o.s1 += cdn * in[2 * (long(sdn) * L.V + here) + 1];
            o.s0 += cup * in[2 * (long(sup) * L.V + here)];
        }
    }
    return o;
}

// Site index i in [0, Ls*V) -> (s, t, x), x fastest (the reference layout).
__device__ __forceinline__ void site_coords(const Lat& L, int i, int& s, int& t, int& x)
{
    s = i / L.V;
    const int r = i - s * L.V;
    t = r / L.Nx;
    x = r - t * L.Nx;
}

// The same operator computed by one thread for one 4-D site (t, x) and every
// fifth-dimension slice: the four link phases are loaded once and reused for
// all Ls slices, and the fifth-dimension hop takes psi(s-1), psi(s), psi(s+1)
// from a rolling register window (each centre spinor is loaded once, as the
// "next" of the previous slice). emit(s, out) receives each output spinor.
template <bool DAG, typename R, typename Emit>
__device__ __forceinline__ void dirac_column(const cplx<R>* __restrict__ in,
                                             const cplx<R>* __restrict__ U, const Lat& L, int t,
                                             int x, Emit emit)
{
    using T = cplx<R>;
    const int Nt = L.Nt, Nx = L.Nx, V = L.V, Ls = L.Ls;
    const int tp = (t + 1 == Nt) ? 0 : t + 1;
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const int here = t * Nx + x;
    const int itp = tp * Nx + x, itm = tm * Nx + x, ixp = t * Nx + xp, ixm = t * Nx + xm;
    const T Ut = U[here];
    const T Utm = U[itm];
    const T Ux = U[V + here];
    const T Uxm = U[V + t * Nx + xm];
    const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
    const R stm = (t == 0) ? R(L.bct) : R(1);
    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    const R dg = R(L.diag), mf = R(L.mf);
    const Spinor<R> first = ld_spinor(in, here);
    Spinor<R> prev = L.fifth ? ld_spinor(in, long(Ls - 1) * V + here) : first;
    Spinor<R> cur = first;
    for (int s = 0; s < Ls; ++s)
    {
        const long sb = long(s) * V;
        const Spinor<R> next = (s + 1 < Ls) ? ld_spinor(in, sb + V + here) : first;
        const Spinor<R> vtp = ld_spinor(in, sb + itp);
        const Spinor<R> vtm = ld_spinor(in, sb + itm);
        const Spinor<R> vxp = ld_spinor(in, sb + ixp);
        const Spinor<R> vxm = ld_spinor(in, sb + ixm);
        T up, lo;
        hop4<DAG, R>(vtp, vtm, vxp, vxm, Ut, Utm, Ux, Uxm, stp, stm, sxp, sxm, up, lo);
        Spinor<R> o{dg * cur.s0 - R(0.5) * up, dg * cur.s1 - R(0.5) * lo};
        if (L.fifth)
        {
            // D: spin 1 from s+1 (m_f psi(0) at the top), spin 0 from s-1 (m_f psi(Ls-1) at 0);
            // D^dag: the directions swapped.
            const R cup = (s + 1 == Ls) ? mf : R(-1);
            const R cdn = (s == 0) ? mf : R(-1);
            if (!DAG)
            {
                o.s1 += cup * next.s1;
                o.s0 += cdn * prev.s0;
            }
            else
            {
                o.s1 += cdn * prev.s1;
                o.s0 += cup * next.s0;
            }
        }
        emit(s, o);
        prev = cur;
        cur = next;
    }
}

}  // namespace dwfb
