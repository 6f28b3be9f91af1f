// Persistent cooperative CG kernels for the Wilson and domain-wall normal
// operators, solving many right-hand sides in one launch.
//
// Work decomposition: every right-hand side is cut into `nch` chunks of `ch`
// sites; a (right-hand side, chunk) pair is one work unit, handed to blocks in
// round-robin order over the right-hand sides still iterating. Each unit
// writes its partial sums to `part`; after the grid barrier every block adds
// the partials of every active right-hand side in the same fixed order, so all
// blocks hold bit-identical scalars (alpha, beta, convergence flags) and take
// the same branches without further communication.
//
// Reference algorithm (DWF_SOLVER_CG64): domain_wall/include/cg_solver.hpp:17-64.
// Per iteration, with A = D2 D1 (D1 = D for D^dag D, D^dag for D D^dag):
//   phase 1: p = r + beta p_old (formed on the fly at every stencil point and
//            stored at the centre into the other direction buffer),
//            t = D1 p, |t|^2 = <p, A p>                     | grid barrier
//   phase 2: x += alpha p, r -= alpha D2 t, |r|^2           | grid barrier
// The direction is double-buffered so that phase 1 reads p_old and r at the
// neighbours while it writes the new p, with no third barrier.
#include "persist.cuh"


namespace dwfb {
using namespace persist;
namespace {
}  // namespace

template <bool FUSED, int MINB>
__global__ void __launch_bounds__(256, MINB) cg64_kernel(SolveDesc d)
{
    const Smem s = carve(d.nrhs);
    for (int j = threadIdx.x; j < d.nrhs; j += blockDim.x)
    {
        s.state[j] = (d.active_in && !d.active_in[j]) ? DWF_OK : RHS_ACTIVE;
        s.iters[j] = 0;
        s.ru[j] = 0;
        s.rr[j] = 0.0;
        s.bb[j] = 0.0;
    }
    __syncthreads();
    const long fs = d.fsz;
    const bool dag1 = d.dag_first != 0;
    int nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });
    if (!init_residual(d, s, nact, false))
        return;
    for (int k = threadIdx.x; k < nact; k += blockDim.x)
    {
        const int j = s.act[k];
        if (s.bb[j] == 0.0 || converged_now(d, s.rr[j], s.bb[j]))
            s.state[j] = DWF_OK;
    }
    __syncthreads();
    nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });

    for (int it = 1; it <= d.maxiter && nact > 0; ++it)
    {
        double2* pc = (FUSED && !(it & 1)) ? d.p2 : d.p;  // direction of this iteration
        const double2* po = (pc == d.p) ? d.p2 : d.p;     // previous direction
        const bool fuse = FUSED && it > 1;
        // phase 1: p = r + beta p_old, t = D1 p, <p, A p> = |t|^2
        sweep(d, s.act, nact, s.scratch, true, [&](int j, int i, long uo) {
            Spinor<double> v;
            if (!fuse)
                v = op_site<double>(d, dag1, pc + j * fs, d.U64 + uo, i);
            else
            {
                const DirLd<double> ld{d.r + j * fs, po + j * fs, s.cf[j]};
                v = op_site_ld<double>(d, dag1, ld, d.U64 + uo, i);
                st_spinor(pc + j * fs, i, ld.sp(i));
            }
            st_spinor(d.t + j * fs, i, v);
            return make_double2(spinor_norm2(v), 0.0);
        });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        reduce_listed(d, s.act, nact, 0, s.aux);
        for (int k = threadIdx.x; k < nact; k += blockDim.x)
        {
            const int j = s.act[k];
            if (s.aux[j] == 0.0)
            {
                s.state[j] = DWF_ZERO_DENOM;  // cg_solver.hpp:45-46
                s.iters[j] = it;
            }
            else
                s.al[j] = s.rr[j] / s.aux[j];
        }
        __syncthreads();
        nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });

        // phase 2: x += alpha p; r -= alpha A p
        sweep(d, s.act, nact, s.scratch, true, [&](int j, int i, long uo) {
            const double a = s.al[j];
            const Spinor<double> ap = op_site<double>(d, !dag1, d.t + j * fs, d.U64 + uo, i);
            const Spinor<double> p = ld_spinor(pc + j * fs, i);
            const Spinor<double> x = ld_spinor(d.x + j * fs, i);
            const Spinor<double> r = ld_spinor(d.r + j * fs, i);
            st_spinor(d.x + j * fs, i, axpy(a, p, x));
            const Spinor<double> rn = axpy(-a, ap, r);
            st_spinor(d.r + j * fs, i, rn);
            return make_double2(spinor_norm2(rn), 0.0);
        });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        reduce_listed(d, s.act, nact, 0, s.aux);
        for (int k = threadIdx.x; k < nact; k += blockDim.x)
        {
            const int j = s.act[k];
            const double rn = s.aux[j];
            s.iters[j] = d.eigen_rule ? it - 1 : it;
            if (converged_now(d, rn, s.bb[j]))
            {
                s.state[j] = DWF_OK;
                s.rr[j] = rn;
            }
            else
            {
                s.iters[j] = it;
                s.cf[j] = rn / s.rr[j];
                s.rr[j] = rn;
            }
        }
        __syncthreads();
        nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });
        if (FUSED)
            continue;
        if (nact == 0)
            break;
        // phase 3: p = r + beta p
        sweep(d, s.act, nact, s.scratch, false, [&](int j, int i, long uo) {
            const Spinor<double> p = ld_spinor(d.p + j * fs, i);
            const Spinor<double> r = ld_spinor(d.r + j * fs, i);
            st_spinor(d.p + j * fs, i, axpy(s.cf[j], p, r));
            return make_double2(0.0, 0.0);
        });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
    }
    write_outputs(d, s);
}

// Mixed precision: FP32 inner CG on (r32, p32, t32) with the correction
// accumulated in e32; a reliable update adds e32 into the FP64 iterate and
// replaces the residual by the FP64 true residual b - A x whenever the FP32
// residual has dropped by `delta` since the last update, or when it claims
// convergence. A right-hand side converges only on the FP64 true residual.
template <bool FUSED, int MINB>
__global__ void __launch_bounds__(256, MINB) cg_mixed_kernel(SolveDesc d)
{
    const Smem s = carve(d.nrhs);
    for (int j = threadIdx.x; j < d.nrhs; j += blockDim.x)
    {
        s.state[j] = (d.active_in && !d.active_in[j]) ? DWF_OK : RHS_ACTIVE;
        s.iters[j] = 0;
        s.ru[j] = 0;
        s.rr[j] = 0.0;
        s.bb[j] = 0.0;
        s.flag[j] = 0;
    }
    __syncthreads();
    const long fs = d.fsz;
    const bool dag1 = d.dag_first != 0;
    int nact = compact(d.nrhs, s.act, s.scratch, [&](int j) { return s.state[j] == RHS_ACTIVE; });
    if (!init_residual(d, s, nact, true))
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
    // stall counters live in the upper bits of flag: flag = 2*stalls + update bit
    for (int it = 1; it <= d.maxiter && nact > 0; ++it)
    {
        float2* pc = (FUSED && !(it & 1)) ? d.p32b : d.p32;
        const float2* po = (pc == d.p32) ? d.p32b : d.p32;
        const bool fuse = FUSED && it > 1;
        sweep(d, s.act, nact, s.scratch, true, [&](int j, int i, long uo) {
            Spinor<float> v;
            if (!fuse)
                v = op_site<float>(d, dag1, pc + j * fs, d.U32 + uo, i);
            else
            {
                const DirLd<float> ld{d.r32 + j * fs, po + j * fs, float(s.cf[j])};
                v = op_site_ld<float>(d, dag1, ld, d.U32 + uo, i);
                st_spinor(pc + j * fs, i, ld.sp(i));
            }
            st_spinor(d.t32 + j * fs, i, v);
            return make_double2(spinor_norm2(v), 0.0);
        });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
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

        sweep(d, s.act, nact, s.scratch, true, [&](int j, int i, long uo) {
            const float a = float(s.al[j]);
            const Spinor<float> ap = op_site<float>(d, !dag1, d.t32 + j * fs, d.U32 + uo, i);
            const Spinor<float> p = ld_spinor(pc + j * fs, i);
            const Spinor<float> e = ld_spinor(d.e32 + j * fs, i);
            const Spinor<float> r = ld_spinor(d.r32 + j * fs, i);
            st_spinor(d.e32 + j * fs, i, axpy(a, p, e));
            const Spinor<float> rn = axpy(-a, ap, r);
            st_spinor(d.r32 + j * fs, i, rn);
            return make_double2(spinor_norm2(rn), 0.0);
        });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
        reduce_listed(d, s.act, nact, 0, s.aux);
        for (int k = threadIdx.x; k < nact; k += blockDim.x)
        {
            const int j = s.act[k];
            const double rn = s.aux[j];
            s.iters[j] = it;
            const bool want = rn < d.delta * d.delta * s.rru[j] || converged_now(d, rn, s.bb[j]) ||
                              it == d.maxiter;
            s.flag[j] = (s.flag[j] & ~1) | (want ? 1 : 0);
            s.cf[j] = rn / s.rr[j];  // beta unless a reliable update replaces it
            s.rr[j] = rn;
        }
        __syncthreads();
        const bool ru_now = d.ru_period <= 1 || it % d.ru_period == 0 || it == d.maxiter;
        const int nru = ru_now ? compact(d.nrhs, s.act, s.scratch, [&](int j) {
            return s.state[j] == RHS_ACTIVE && (s.flag[j] & 1);
        }) : 0;
        if (nru > 0)
        {
            // Reliable update, part 1: t = D1 (x + e) in FP64, with x + e
            // formed on the fly from its neighbourhood and parked in r.
            sweep(d, s.act, nru, s.scratch, false, [&](int j, int i, long uo) {
                int ss, tt, xx;
                site_coords(d.L, i, ss, tt, xx);
                const SumLd xe{d.x + j * fs, d.e32 + j * fs};
                const Spinor<double> v =
                    dag1 ? dirac_site_ld<true, double>(xe, d.U64 + uo, d.L, ss, tt, xx)
                         : dirac_site_ld<false, double>(xe, d.U64 + uo, d.L, ss, tt, xx);
                st_spinor(d.t + j * fs, i, v);
                st_spinor(d.r + j * fs, i, xe.sp(i));
                return make_double2(0.0, 0.0);
            });
            if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
                return;
            // part 2: x = x + e; r = b - D2 t; r32 = r; e = 0
            sweep(d, s.act, nru, s.scratch, true, [&](int j, int i, long uo) {
                const Spinor<double> xn = ld_spinor(d.r + j * fs, i);
                const Spinor<double> a = op_site<double>(d, !dag1, d.t + j * fs, d.U64 + uo, i);
                const Spinor<double> b = ld_spinor(d.b + j * fs, i);
                st_spinor(d.x + j * fs, i, xn);
                const Spinor<double> r = {b.s0 - a.s0, b.s1 - a.s1};
                st_spinor(d.r + j * fs, i, r);
                st_spinor(d.r32 + j * fs, i, to32(r));
                st_spinor(d.e32 + j * fs, i,
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
                // beta = |r_new|^2 / |r_old|^2 with the replaced residual
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
        if (FUSED)
            continue;
        if (nact == 0)
            break;
        sweep(d, s.act, nact, s.scratch, false, [&](int j, int i, long uo) {
            const Spinor<float> p = ld_spinor(d.p32 + j * fs, i);
            const Spinor<float> r = ld_spinor(d.r32 + j * fs, i);
            st_spinor(d.p32 + j * fs, i, axpy(float(s.cf[j]), p, r));
            return make_double2(0.0, 0.0);
        });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return;
    }
    write_outputs(d, s);
}

// Instances: the fused two-barrier form at two blocks per SM wins when a
// single right-hand side is latency bound; the three-barrier form at three
// blocks per SM wins for batches (fewer loads per site).
template __global__ void cg64_kernel<true, 2>(SolveDesc);
template __global__ void cg64_kernel<false, 3>(SolveDesc);
template __global__ void cg_mixed_kernel<true, 2>(SolveDesc);
template __global__ void cg_mixed_kernel<false, 3>(SolveDesc);

}  // namespace dwfb
