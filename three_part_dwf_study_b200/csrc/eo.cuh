// Even-odd (checkerboard) preconditioning of the domain-wall operator.
//
// With M5 the part of D that is local in the 4-D site (the diagonal 3 - M5 and
// the fifth-dimension hop) and H the 4-D hop term, D = M5 + H couples only
// opposite 4-D parities through H. On odd sites the Schur complement is
//   Dhat = M5 - H_oe M5^-1 H_eo,   Dhat^dag = M5^dag - H^dag_oe M5^dag^-1 H^dag_eo,
// and D x = b becomes Dhat x_o = b_o - H_oe M5^-1 b_e, x_e = M5^-1 (b_e - H_eo x_o).
//
// Parity fields: site (s, t, x) with (t + x) % 2 == parity is stored at
// s*Vh + t*Nxh + x/2 (Vh = Nt*Nx/2, Nxh = Nx/2); Nt and Nx must be even. The
// t +- 1 neighbours of (t, x) keep x, the x +- 1 neighbours are at
// (x +- 1)/2, all in the other parity's field.
//
// M5 acts per 4-D site and per spin as an Ls x Ls matrix (c = 3 - M5):
//   "up" form   (Y y)(s) = c y(s) - y(s+1),  (Y y)(Ls-1) = c y(Ls-1) + m_f y(0)
//   "down" form (Z y)(s) = c y(s) - y(s-1),  (Z y)(0)    = c y(0)    + m_f y(Ls-1)
// D uses Y on spin 1 and Z on spin 0 (dwf_operator.hpp:71-86); D^dag the other
// way round (:150-165). Their inverses in closed form, stable for c >= 1:
//   Y^-1: y(0) = S/(1 + m_f c^-Ls), S = sum_k z(k) c^-(k+1);
//         y(Ls-1) = (z(Ls-1) - m_f y(0))/c, y(s) = (z(s) + y(s+1))/c downwards
//   Z^-1: y(Ls-1) = S/(1 + m_f c^-Ls), S = sum_k z(k) c^-(Ls-k);
//         y(0) = (z(0) - m_f y(Ls-1))/c, y(s) = (z(s) + y(s-1))/c upwards.
#pragma once

#include "dirac.cuh"
#include "solver.cuh"

namespace dwfb {

struct EoGeo
{
    int Nxh, Vh;
};

// Launch descriptor of the persistent even-odd solver kernel.
struct EoDesc
{
    SolveDesc d;    // fields are parity fields (fsz = 2*Vh*Ls); d.nch/d.ch chunk 5-D odd sites
    EoGeo g;
    int nch4, ch4;  // chunking of the 4-D even sites
    double2* y64;   // even temporaries
    float2* y32;
    double2* xn64;  // reliable update: x + e parked here
    int zsmem;      // 1: the FP32 hop + M5^-1 phases keep the slices in shared memory
    unsigned long long* phase_ns;  // optional [16]: per-phase ns [0, 8) and counts [8, 16)
};

// Hop term H (DAG = false) or H^dag of the site (s, t, x), reading the other
// parity's field through `in`: -1/2 sum_mu [...] (the 4-D part of dirac_site).
template <bool DAG, typename R, typename Ld>
__device__ __forceinline__ Spinor<R> eo_hop(const Ld& in, const cplx<R>* __restrict__ U,
                                            const Lat& L, EoGeo g, int s, int t, int x)
{
    using T = cplx<R>;
    const int Nt = L.Nt, Nx = L.Nx;
    const int tp = (t + 1 == Nt) ? 0 : t + 1;
    const int tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1;
    const int xm = (x == 0) ? Nx - 1 : x - 1;
    const long sb = long(s) * g.Vh;
    const Spinor<R> vtp = in.sp(sb + tp * g.Nxh + (x >> 1));
    const Spinor<R> vtm = in.sp(sb + tm * g.Nxh + (x >> 1));
    const Spinor<R> vxp = in.sp(sb + t * g.Nxh + (xp >> 1));
    const Spinor<R> vxm = in.sp(sb + t * g.Nxh + (xm >> 1));
    const int here = t * Nx + x;
    const T Ut = U[here];
    const T Utm = U[tm * Nx + x];
    const T Ux = U[L.V + here];
    const T Uxm = U[L.V + t * Nx + xm];
    const R stp = (t == Nt - 1) ? R(L.bct) : R(1);
    const R stm = (t == 0) ? R(L.bct) : R(1);
    const R sxp = (x == Nx - 1) ? R(L.bcx) : R(1);
    const R sxm = (x == 0) ? R(L.bcx) : R(1);
    constexpr R kf = DAG ? R(1) : R(-1);
    constexpr R kb = -kf;
    T w = cmul(Ut, stp * (vtp.s0 + kf * vtp.s1));
    T up = w;
    T lo = kf * w;
    w = cmulc(Utm, stm * (vtm.s0 + kb * vtm.s1));
    up += w;
    lo += kb * w;
    w = cmul(Ux, sxp * (vxp.s0 - kf * itimes(vxp.s1)));
    up += w;
    lo += kf * itimes(w);
    w = cmulc(Uxm, sxm * (vxm.s0 - kb * itimes(vxm.s1)));
    up += w;
    lo += kb * itimes(w);
    return {R(-0.5) * up, R(-0.5) * lo};
}

// eo_hop at a fixed 4-D site for any slice: the neighbour offsets within a
// parity slice and the four links (boundary signs folded in, exact for signs
// +-1) are computed once, so a loop over the Ls slices only loads spinors.
template <bool DAG, typename R>
struct EoHopSite
{
    cplx<R> ut, utm, ux, uxm;
    int otp, otm, oxp, oxm;
    __device__ __forceinline__ EoHopSite(const cplx<R>* __restrict__ U, const Lat& L, EoGeo g,
                                         int t, int x)
    {
        const int Nt = L.Nt, Nx = L.Nx;
        const int tp = (t + 1 == Nt) ? 0 : t + 1;
        const int tm = (t == 0) ? Nt - 1 : t - 1;
        const int xp = (x + 1 == Nx) ? 0 : x + 1;
        const int xm = (x == 0) ? Nx - 1 : x - 1;
        otp = tp * g.Nxh + (x >> 1);
        otm = tm * g.Nxh + (x >> 1);
        oxp = t * g.Nxh + (xp >> 1);
        oxm = t * g.Nxh + (xm >> 1);
        const int here = t * Nx + x;
        ut = ((t == Nt - 1) ? R(L.bct) : R(1)) * U[here];
        utm = ((t == 0) ? R(L.bct) : R(1)) * U[tm * Nx + x];
        ux = ((x == Nx - 1) ? R(L.bcx) : R(1)) * U[L.V + here];
        uxm = ((x == 0) ? R(L.bcx) : R(1)) * U[L.V + t * Nx + xm];
    }
    template <typename Ld>
    __device__ __forceinline__ Spinor<R> at(const Ld& in, long sb) const
    {
        using T = cplx<R>;
        constexpr R kf = DAG ? R(1) : R(-1);
        constexpr R kb = -kf;
        const Spinor<R> vtp = in.sp(sb + otp);
        const Spinor<R> vtm = in.sp(sb + otm);
        const Spinor<R> vxp = in.sp(sb + oxp);
        const Spinor<R> vxm = in.sp(sb + oxm);
        T w = cmul(ut, vtp.s0 + kf * vtp.s1);
        T up = w;
        T lo = kf * w;
        w = cmulc(utm, vtm.s0 + kb * vtm.s1);
        up += w;
        lo += kb * w;
        w = cmul(ux, vxp.s0 - kf * itimes(vxp.s1));
        up += w;
        lo += kf * itimes(w);
        w = cmulc(uxm, vxm.s0 - kb * itimes(vxm.s1));
        up += w;
        lo += kb * itimes(w);
        return {R(-0.5) * up, R(-0.5) * lo};
    }
};

// M5 (DAG = false) or M5^dag at slice s of the 4-D site h of a parity field.
template <bool DAG, typename R, typename Ld>
__device__ __forceinline__ Spinor<R> eo_m5(const Ld& in, const Lat& L, EoGeo g, int s, int h)
{
    const Spinor<R> c = in.sp(long(s) * g.Vh + h);
    const R dg = R(L.diag);
    Spinor<R> o{dg * c.s0, dg * c.s1};
    const int Ls = L.Ls;
    const int sup = (s + 1 == Ls) ? 0 : s + 1;
    const R cup = (s + 1 == Ls) ? R(L.mf) : R(-1);
    const int sdn = (s == 0) ? Ls - 1 : s - 1;
    const R cdn = (s == 0) ? R(L.mf) : R(-1);
    if (!DAG)
    {
        o.s1 += cup * in.c(2 * (long(sup) * g.Vh + h) + 1);
        o.s0 += cdn * in.c(2 * (long(sdn) * g.Vh + h));
    }
    else
    {
        o.s1 += cdn * in.c(2 * (long(sdn) * g.Vh + h) + 1);
        o.s0 += cup * in.c(2 * (long(sup) * g.Vh + h));
    }
    return o;
}

// out(:, h) = M5^-1 [src(:, h) + sgn * H in (:, h)] for the 4-D site (t, k) of
// parity po (M5^dag^-1 and H^dag when DAG). `in` may be absent (has_in =
// false) and src may be null. Two passes over s on this thread's own column
// of `out`: the first stores z and accumulates the closed-form sums, the
// second runs the recurrences in place.
template <bool DAG, typename R, typename Ld>
__device__ __forceinline__ void eo_hopinv_site(const Ld& in, bool has_in,
                                               const cplx<R>* __restrict__ src, R sgn,
                                               cplx<R>* __restrict__ out,
                                               const cplx<R>* __restrict__ U, const Lat& L,
                                               EoGeo g, int t, int k, int po)
{
    using T = cplx<R>;
    const int x = 2 * k + ((t + po) & 1);
    const int h = t * g.Nxh + k;
    const int Ls = L.Ls;
    const R c = R(L.diag), ci = R(1) / c, mf = R(L.mf);
    // D: spin 1 up form, spin 0 down form; D^dag: the other way round.
    T s_up = mkc(R(0), R(0)), s_dn = mkc(R(0), R(0));
    R pw = ci;  // c^-(s+1)
    R cmls = R(1);
    for (int s = 0; s < Ls; ++s)
    {
        Spinor<R> z{mkc(R(0), R(0)), mkc(R(0), R(0))};
        if (src)
            z = ld_spinor(src, long(s) * g.Vh + h);
        if (has_in)
        {
            const Spinor<R> hv = eo_hop<DAG, R>(in, U, L, g, s, t, x);
            z.s0 += sgn * hv.s0;
            z.s1 += sgn * hv.s1;
        }
        st_spinor(out, long(s) * g.Vh + h, z);
        const T zu = DAG ? z.s0 : z.s1;  // component in the up form
        const T zd = DAG ? z.s1 : z.s0;  // component in the down form
        s_up += pw * zu;
        s_dn = ci * (s_dn + zd);  // Horner: sum_k z(k) c^-(Ls-k)
        pw *= ci;
        cmls *= ci;
    }
    const R den = R(1) / (R(1) + mf * cmls);
    const int cu = DAG ? 0 : 1;  // spin component in the up form
    const int cd = 1 - cu;
    // up form: y(Ls-1) from y(0), then downwards
    {
        const T y0 = den * s_up;
        const long i_last = 2 * (long(Ls - 1) * g.Vh + h) + cu;
        T y = ci * (out[i_last] - mf * y0);
        out[i_last] = y;
        for (int s = Ls - 2; s >= 0; --s)
        {
            const long i = 2 * (long(s) * g.Vh + h) + cu;
            y = ci * (out[i] + y);
            out[i] = y;
        }
    }
    // down form: y(0) from y(Ls-1), then upwards
    {
        const T yl = den * s_dn;
        const long i0 = 2 * long(h) + cd;
        T y = ci * (out[i0] - mf * yl);
        out[i0] = y;
        for (int s = 1; s < Ls; ++s)
        {
            const long i = 2 * (long(s) * g.Vh + h) + cd;
            y = ci * (out[i] + y);
            out[i] = y;
        }
    }
}

// Same as eo_hopinv_site with the Ls slices of this thread's column kept in
// shared memory (zs[s * zstride], this thread's own slots) while the two
// recurrences run, so `out` is written once per slice instead of being read
// and rewritten in the serial fifth-dimension sweeps.
template <bool DAG, typename R, typename Ld>
__device__ __forceinline__ void eo_hopinv_site_smem(const Ld& in, cplx<R>* __restrict__ out,
                                                    const cplx<R>* __restrict__ U, const Lat& L,
                                                    EoGeo g, int t, int k, int po,
                                                    Spinor<R>* zs, int zstride)
{
    using T = cplx<R>;
    const int x = 2 * k + ((t + po) & 1);
    const int h = t * g.Nxh + k;
    const int Ls = L.Ls;
    const R c = R(L.diag), ci = R(1) / c, mf = R(L.mf);
    T s_up = mkc(R(0), R(0)), s_dn = mkc(R(0), R(0));
    R pw = ci;
    R cmls = R(1);
    const EoHopSite<DAG, R> hs(U, L, g, t, x);
    // unrolled so that several slices' neighbour loads are in flight together
#pragma unroll 4
    for (int s = 0; s < Ls; ++s)
    {
        const Spinor<R> hv = hs.at(in, long(s) * g.Vh);
        zs[s * zstride] = hv;
        const T zu = DAG ? hv.s0 : hv.s1;
        const T zd = DAG ? hv.s1 : hv.s0;
        s_up += pw * zu;
        s_dn = ci * (s_dn + zd);
        pw *= ci;
        cmls *= ci;
    }
    const R den = R(1) / (R(1) + mf * cmls);
    // up form (spin component DAG ? 0 : 1): y(Ls-1) from y(0), then downwards
    {
        const T y0 = den * s_up;
        Spinor<R>& zl = zs[(Ls - 1) * zstride];
        T y = ci * ((DAG ? zl.s0 : zl.s1) - mf * y0);
        (DAG ? zl.s0 : zl.s1) = y;
        for (int s = Ls - 2; s >= 0; --s)
        {
            Spinor<R>& z = zs[s * zstride];
            y = ci * ((DAG ? z.s0 : z.s1) + y);
            (DAG ? z.s0 : z.s1) = y;
        }
    }
    // down form (the other component): y(0) from y(Ls-1), then upwards
    {
        const T yl = den * s_dn;
        Spinor<R>& z0 = zs[0];
        T y = ci * ((DAG ? z0.s1 : z0.s0) - mf * yl);
        (DAG ? z0.s1 : z0.s0) = y;
        for (int s = 1; s < Ls; ++s)
        {
            Spinor<R>& z = zs[s * zstride];
            y = ci * ((DAG ? z.s1 : z.s0) + y);
            (DAG ? z.s1 : z.s0) = y;
        }
    }
    for (int s = 0; s < Ls; ++s)
        st_spinor(out, long(s) * g.Vh + h, zs[s * zstride]);
}

// 5-D site (s, h) of parity q: a + M5 m - H y (M5^dag, H^dag when DAG); any
// of a, m, y may be absent.
template <bool DAG, typename R, typename LdA, typename LdM, typename LdY>
__device__ __forceinline__ Spinor<R> eo_combine_site(const LdA& a, bool has_a, const LdM& m,
                                                     bool has_m, const LdY& y, bool has_y,
                                                     const cplx<R>* __restrict__ U, const Lat& L,
                                                     EoGeo g, int s, int h, int q)
{
    Spinor<R> o{mkc(R(0), R(0)), mkc(R(0), R(0))};
    if (has_a)
        o = a.sp(long(s) * g.Vh + h);
    if (has_m)
    {
        const Spinor<R> v = eo_m5<DAG, R>(m, L, g, s, h);
        o.s0 += v.s0;
        o.s1 += v.s1;
    }
    if (has_y)
    {
        const int t = h / g.Nxh, k = h - t * g.Nxh;
        const int x = 2 * k + ((t + q) & 1);
        const Spinor<R> v = eo_hop<DAG, R>(y, U, L, g, s, t, x);
        o.s0 = o.s0 - v.s0;
        o.s1 = o.s1 - v.s1;
    }
    return o;
}

}  // namespace dwfb
