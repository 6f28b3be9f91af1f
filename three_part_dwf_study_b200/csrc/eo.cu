// Even-odd preconditioned propagator solve: kernels and the persistent
// mixed-precision CG on the Schur normal operator Dhat^dag Dhat (odd sites).
//
// Per iteration (FP32, c = the right-hand side's links):
//   P1 (4-D even sites)  y = M5^-1 H_eo p
//   P2 (5-D odd sites)   t = M5 p - H_oe y,               |t|^2   | barrier
//   P3 (4-D even sites)  y = M5^dag^-1 H^dag_eo t                  | barrier
//   P4 (5-D odd sites)   Ap = M5^dag t - H^dag_oe y; e += alpha p; r -= alpha Ap, |r|^2 | barrier
//   P5 (5-D odd sites)   p = r + beta p                          | barrier
// (P1 follows P5 of the previous iteration after its barrier.) Reliable
// updates recompute the FP64 residual of the Schur normal equation from
// x + e with the same four operator phases in FP64.
#include <algorithm>
#include <vector>

#include "context.cuh"
#include "eo.cuh"
#include "persist.cuh"

namespace dwfb {

using namespace persist;

namespace {

constexpr int kEven = 0, kOdd = 1;

// Phase timer (block 0, thread 0; only when a phase buffer is given): adds the
// time since the previous mark to slot k. Phases: 0 P1, 1 P2, 2 the alpha
// reduction, 3 P3, 4 P4, 5 the beta reduction and reliable updates, 6 P5, each
// including the grid barrier that ends it.
__device__ __forceinline__ void phase_mark(unsigned long long* ph, int k, unsigned long long& t)
{
    if (ph && blockIdx.x == 0 && threadIdx.x == 0)
    {
        const unsigned long long n = globaltimer_ns();
        ph[k] += n - t;
        ph[8 + k] += 1;
        t = n;
    }
}

template <typename R>
struct NoLd
{
    __device__ __forceinline__ Spinor<R> sp(long) const { return {}; }
    __device__ __forceinline__ cplx<R> c(long) const { return {}; }
};

}  // namespace

// ---- standalone FP64 kernels (set-up and reconstruction) ------------------

__global__ void eo_pack_kernel(Lat L, EoGeo g, const double2* __restrict__ full,
                               double2* __restrict__ ev, double2* __restrict__ od, long nrhs)
{
    const long total = nrhs * L.nsite;
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < total;
         idx += long(gridDim.x) * blockDim.x)
    {
        const long j = idx / L.nsite;
        const int i = int(idx - j * L.nsite);
        int s, t, x;
        site_coords(L, i, s, t, x);
        const long hs = j * g.Vh * L.Ls + long(s) * g.Vh + t * g.Nxh + (x >> 1);
        const Spinor<double> v = ld_spinor(full, idx);
        st_spinor(((t + x) & 1) ? od : ev, hs, v);
    }
}

__global__ void eo_unpack_kernel(Lat L, EoGeo g, const double2* __restrict__ ev,
                                 const double2* __restrict__ od, double2* __restrict__ full,
                                 long nrhs)
{
    const long total = nrhs * L.nsite;
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < total;
         idx += long(gridDim.x) * blockDim.x)
    {
        const long j = idx / L.nsite;
        const int i = int(idx - j * L.nsite);
        int s, t, x;
        site_coords(L, i, s, t, x);
        const long hs = j * g.Vh * L.Ls + long(s) * g.Vh + t * g.Nxh + (x >> 1);
        st_spinor(full, idx, ld_spinor(((t + x) & 1) ? od : ev, hs));
    }
}

// out_even = M5^-1 [src_even + sgn H_eo in_odd] (DAG: the D^dag forms), one
// thread per (rhs, 4-D even site).
template <bool DAG>
__global__ void eo_hopinv_kernel(Lat L, EoGeo g, const double2* __restrict__ in,
                                 const double2* __restrict__ src, double sgn,
                                 double2* __restrict__ out, const double2* __restrict__ U,
                                 long usz, const int* __restrict__ conf, long nrhs)
{
    const long fh = 2L * g.Vh * L.Ls;
    const long total = nrhs * g.Vh;
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < total;
         idx += long(gridDim.x) * blockDim.x)
    {
        const long j = idx / g.Vh;
        const int h = int(idx - j * g.Vh);
        const int t = h / g.Nxh, k = h - t * g.Nxh;
        const FieldLd<double> ld{in ? in + j * fh : nullptr};
        eo_hopinv_site<DAG, double>(ld, in != nullptr, src ? src + j * fh : nullptr, sgn,
                                    out + j * fh, U + long(conf[j]) * usz, L, g, t, k, kEven);
    }
}

// out_odd = a + M5 m - H_oe y_even (DAG: the D^dag forms), one thread per
// (rhs, 5-D odd site).
template <bool DAG>
__global__ void eo_combine_kernel(Lat L, EoGeo g, const double2* __restrict__ a,
                                  const double2* __restrict__ m, const double2* __restrict__ y,
                                  double2* __restrict__ out, const double2* __restrict__ U,
                                  long usz, const int* __restrict__ conf, long nrhs)
{
    const long fh = 2L * g.Vh * L.Ls;
    const long per = long(g.Vh) * L.Ls;
    const long total = nrhs * per;
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < total;
         idx += long(gridDim.x) * blockDim.x)
    {
        const long j = idx / per;
        const int i = int(idx - j * per);
        const int s = i / g.Vh, h = i - s * g.Vh;
        const FieldLd<double> la{a ? a + j * fh : nullptr}, lm{m ? m + j * fh : nullptr},
            ly{y ? y + j * fh : nullptr};
        st_spinor(out + j * fh, i,
                  eo_combine_site<DAG, double>(la, a != nullptr, lm, m != nullptr, ly,
                                               y != nullptr, U + long(conf[j]) * usz, L, g, s,
                                               h, kOdd));
    }
}

template __global__ void eo_hopinv_kernel<false>(Lat, EoGeo, const double2*, const double2*,
                                                 double, double2*, const double2*, long,
                                                 const int*, long);
template __global__ void eo_hopinv_kernel<true>(Lat, EoGeo, const double2*, const double2*,
                                                double, double2*, const double2*, long,
                                                const int*, long);
template __global__ void eo_combine_kernel<false>(Lat, EoGeo, const double2*, const double2*,
                                                  const double2*, double2*, const double2*, long,
                                                  const int*, long);
template __global__ void eo_combine_kernel<true>(Lat, EoGeo, const double2*, const double2*,
                                                 const double2*, double2*, const double2*, long,
                                                 const int*, long);

// ---- persistent mixed-precision Schur CG ------------------------------------

#ifndef DWFB_EO_MINB
#define DWFB_EO_MINB 2  // resident 256-thread blocks per SM the register budget targets (2: no spills)
#endif

__global__ void __launch_bounds__(256, DWFB_EO_MINB) cg_eo_mixed_kernel(EoDesc e)
{
    const SolveDesc& d = e.d;
    const EoGeo g = e.g;
    const Smem s = carve(d.nrhs);
    for (int j = threadIdx.x; j < d.nrhs; j += blockDim.x)
    {
        s.state[j] = RHS_ACTIVE;
        s.iters[j] = 0;
        s.ru[j] = 0;
        s.rr[j] = 0.0;
        s.bb[j] = 0.0;
        s.flag[j] = 0;
    }
    __syncthreads();
    const long fs = d.fsz;
    int nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });
    if (!init_residual(d, s, nact, true))  // x = 0: r = b, r32 = p32 = r, e32 = 0
        return;
    for (int k = threadIdx.x; k < nact; k += blockDim.x)
    {
        const int j = s.act[k];
        s.rru[j] = s.rr[j];
        if (s.bb[j] == 0.0 || converged_now(d, s.rr[j], s.bb[j]))
            s.state[j] = DWF_OK;
    }
    __syncthreads();
    nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });
    const int nsite4 = g.Vh, nsite5 = g.Vh * d.L.Ls;
    const long fh = fs;
    // per-thread slice columns for the FP32 hop + M5^-1 phases (after the
    // solver's own shared memory, 16-byte aligned)
    extern __shared__ double sm_all[];
    Spinor<float>* zs = reinterpret_cast<Spinor<float>*>(
        reinterpret_cast<char*>(sm_all) + ((solver_smem_bytes(d.nrhs) + 15) & ~size_t(15))) + threadIdx.x;

    unsigned long long ph_t = globaltimer_ns();
    for (int it = 1; it <= d.maxiter && nact > 0; ++it)
    {
        // P1: y = M5^-1 H_eo p
        sweep_sites(d, s.act, nact, nsite4, e.nch4, e.ch4, s.scratch, false,
                    [&](int j, int h, long uo) {
                        const int t = h / g.Nxh, k = h - t * g.Nxh;
                        if (e.zsmem)
                            eo_hopinv_site_smem<false, float>(FieldLd<float>{d.p32 + j * fh},
                                                              e.y32 + j * fh, d.U32 + uo, d.L, g,
                                                              t, k, kEven, zs, blockDim.x);
                        else
                            eo_hopinv_site<false, float>(FieldLd<float>{d.p32 + j * fh}, true,
                                                         nullptr, 1.0f, e.y32 + j * fh,
                                                         d.U32 + uo, d.L, g, t, k, kEven);
                        return make_double2(0.0, 0.0);
                    });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        phase_mark(e.phase_ns, 0, ph_t);
        // P2: t = M5 p - H_oe y, |t|^2
        sweep_sites(d, s.act, nact, nsite5, d.nch, d.ch, s.scratch, true,
                    [&](int j, int i, long uo) {
                        const int ss = i / g.Vh, h = i - ss * g.Vh;
                        const Spinor<float> v = eo_combine_site<false, float>(
                            NoLd<float>{}, false, FieldLd<float>{d.p32 + j * fh}, true,
                            FieldLd<float>{e.y32 + j * fh}, true, d.U32 + uo, d.L, g, ss, h,
                            kOdd);
                        st_spinor(d.t32 + j * fh, i, v);
                        return make_double2(spinor_norm2(v), 0.0);
                    });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        phase_mark(e.phase_ns, 1, ph_t);
        reduce_listed(d, s.act, nact, 0, s.aux);
        for (int k = threadIdx.x; k < nact; k += blockDim.x)
        {
            const int j = s.act[k];
            if (s.aux[j] == 0.0 || !isfinite(s.aux[j]))
            {
                s.state[j] = DWF_NOT_CONVERGED;
                s.iters[j] = it;
            }
            else
                s.al[j] = s.rr[j] / s.aux[j];
        }
        __syncthreads();
        nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });
        phase_mark(e.phase_ns, 2, ph_t);
        // P3: y = M5^dag^-1 H^dag_eo t
        sweep_sites(d, s.act, nact, nsite4, e.nch4, e.ch4, s.scratch, false,
                    [&](int j, int h, long uo) {
                        const int t = h / g.Nxh, k = h - t * g.Nxh;
                        if (e.zsmem)
                            eo_hopinv_site_smem<true, float>(FieldLd<float>{d.t32 + j * fh},
                                                             e.y32 + j * fh, d.U32 + uo, d.L, g,
                                                             t, k, kEven, zs, blockDim.x);
                        else
                            eo_hopinv_site<true, float>(FieldLd<float>{d.t32 + j * fh}, true,
                                                        nullptr, 1.0f, e.y32 + j * fh, d.U32 + uo,
                                                        d.L, g, t, k, kEven);
                        return make_double2(0.0, 0.0);
                    });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        phase_mark(e.phase_ns, 3, ph_t);
        // P4: Ap = M5^dag t - H^dag_oe y; e += alpha p; r -= alpha Ap
        sweep_sites(d, s.act, nact, nsite5, d.nch, d.ch, s.scratch, true,
                    [&](int j, int i, long uo) {
                        const int ss = i / g.Vh, h = i - ss * g.Vh;
                        const float a = float(s.al[j]);
                        const Spinor<float> ap = eo_combine_site<true, float>(
                            NoLd<float>{}, false, FieldLd<float>{d.t32 + j * fh}, true,
                            FieldLd<float>{e.y32 + j * fh}, true, d.U32 + uo, d.L, g, ss, h,
                            kOdd);
                        const Spinor<float> p = ld_spinor(d.p32 + j * fh, i);
                        const Spinor<float> ee = ld_spinor(d.e32 + j * fh, i);
                        const Spinor<float> r = ld_spinor(d.r32 + j * fh, i);
                        st_spinor(d.e32 + j * fh, i, axpy(a, p, ee));
                        const Spinor<float> rn = axpy(-a, ap, r);
                        st_spinor(d.r32 + j * fh, i, rn);
                        return make_double2(spinor_norm2(rn), 0.0);
                    });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        phase_mark(e.phase_ns, 4, ph_t);
        reduce_listed(d, s.act, nact, 0, s.aux);
        for (int k = threadIdx.x; k < nact; k += blockDim.x)
        {
            const int j = s.act[k];
            const double rn = s.aux[j];
            s.iters[j] = it;
            const bool want = rn < d.delta * d.delta * s.rru[j] || converged_now(d, rn, s.bb[j]) ||
                              it == d.maxiter;
            s.flag[j] = (s.flag[j] & ~1) | (want ? 1 : 0);
            s.cf[j] = rn / s.rr[j];
            s.rr[j] = rn;
        }
        __syncthreads();
        const bool ru_now = d.ru_period <= 1 || it % d.ru_period == 0 || it == d.maxiter;
        const int nru = ru_now ? compact(d.nrhs, s.act, s.scratch, [&](int j) {
            return s.state[j] == RHS_ACTIVE && (s.flag[j] & 1);
        }) : 0;
        if (nru > 0)
        {
            // FP64 residual of the Schur normal equation at x + e:
            // (a) y64 = M5^-1 H_eo (x + e)
            sweep_sites(d, s.act, nru, nsite4, e.nch4, e.ch4, s.scratch, false,
                        [&](int j, int h, long uo) {
                            const int t = h / g.Nxh, k = h - t * g.Nxh;
                            eo_hopinv_site<false, double>(SumLd{d.x + j * fh, d.e32 + j * fh},
                                                          true, nullptr, 1.0, e.y64 + j * fh,
                                                          d.U64 + uo, d.L, g, t, k, kEven);
                            return make_double2(0.0, 0.0);
                        });
            if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
                return;
            // (b) t64 = M5 (x + e) - H_oe y64; park x + e in xn64
            sweep_sites(d, s.act, nru, nsite5, d.nch, d.ch, s.scratch, false,
                        [&](int j, int i, long uo) {
                            const int ss = i / g.Vh, h = i - ss * g.Vh;
                            const SumLd xe{d.x + j * fh, d.e32 + j * fh};
                            const Spinor<double> v = eo_combine_site<false, double>(
                                NoLd<double>{}, false, xe, true, FieldLd<double>{e.y64 + j * fh},
                                true, d.U64 + uo, d.L, g, ss, h, kOdd);
                            st_spinor(d.t + j * fh, i, v);
                            st_spinor(e.xn64 + j * fh, i, xe.sp(i));
                            return make_double2(0.0, 0.0);
                        });
            if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
                return;
            // (c) y64 = M5^dag^-1 H^dag_eo t64
            sweep_sites(d, s.act, nru, nsite4, e.nch4, e.ch4, s.scratch, false,
                        [&](int j, int h, long uo) {
                            const int t = h / g.Nxh, k = h - t * g.Nxh;
                            eo_hopinv_site<true, double>(FieldLd<double>{d.t + j * fh}, true,
                                                         nullptr, 1.0, e.y64 + j * fh,
                                                         d.U64 + uo, d.L, g, t, k, kEven);
                            return make_double2(0.0, 0.0);
                        });
            if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
                return;
            // (d) r = b - (M5^dag t64 - H^dag_oe y64); x = x + e; r32 = r; e = 0
            sweep_sites(d, s.act, nru, nsite5, d.nch, d.ch, s.scratch, true,
                        [&](int j, int i, long uo) {
                            const int ss = i / g.Vh, h = i - ss * g.Vh;
                            const Spinor<double> a = eo_combine_site<true, double>(
                                NoLd<double>{}, false, FieldLd<double>{d.t + j * fh}, true,
                                FieldLd<double>{e.y64 + j * fh}, true, d.U64 + uo, d.L, g, ss, h,
                                kOdd);
                            const Spinor<double> b = ld_spinor(d.b + j * fh, i);
                            const Spinor<double> r = {b.s0 - a.s0, b.s1 - a.s1};
                            st_spinor(d.x + j * fh, i, ld_spinor(e.xn64 + j * fh, i));
                            st_spinor(d.r + j * fh, i, r);
                            st_spinor(d.r32 + j * fh, i, to32(r));
                            st_spinor(d.e32 + j * fh, i,
                                      Spinor<float>{make_float2(0.f, 0.f), make_float2(0.f, 0.f)});
                            return make_double2(spinor_norm2(r), 0.0);
                        });
            if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
                return;
            reduce_listed(d, s.act, nru, 0, s.aux);
            for (int k = threadIdx.x; k < nru; k += blockDim.x)
            {
                const int j = s.act[k];
                const double rt = s.aux[j];
                s.ru[j] += 1;
                s.cf[j] = s.cf[j] * (rt / s.rr[j]);
                const int stalls = (rt >= 0.5 * s.rru[j]) ? (s.flag[j] >> 1) + 1 : 0;
                s.flag[j] = stalls << 1;
                s.rr[j] = rt;
                s.rru[j] = rt;
                if (converged_now(d, rt, s.bb[j]))
                    s.state[j] = DWF_OK;
                else if (!isfinite(rt) || stalls >= d.stall_limit || it == d.maxiter)
                    s.state[j] = DWF_NOT_CONVERGED;
            }
            __syncthreads();
        }
        nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });
        if (nact == 0)
            break;
        phase_mark(e.phase_ns, 5, ph_t);
        // P5: p = r + beta p
        sweep_sites(d, s.act, nact, nsite5, d.nch, d.ch, s.scratch, false,
                    [&](int j, int i, long uo) {
                        const Spinor<float> p = ld_spinor(d.p32 + j * fh, i);
                        const Spinor<float> r = ld_spinor(d.r32 + j * fh, i);
                        st_spinor(d.p32 + j * fh, i, axpy(float(s.cf[j]), p, r));
                        return make_double2(0.0, 0.0);
                    });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        phase_mark(e.phase_ns, 6, ph_t);
    }
    write_outputs(d, s);
}

}  // namespace dwfb
