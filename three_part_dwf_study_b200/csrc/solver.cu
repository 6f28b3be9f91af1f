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
#include "solver.cuh"


namespace dwfb {
namespace {

struct Smem
{
    double* scratch;  // 64 doubles
    double* rr;       // |r|^2 per right-hand side
    double* bb;       // |b|^2
    double* cf;       // beta
    double* al;       // alpha
    double* aux;      // reduction target
    double* rru;      // |r|^2 at the last reliable update (mixed)
    int* state;       // RHS_ACTIVE or the final dwf_status
    int* iters;
    int* act;         // compacted list of active right-hand sides
    int* ru;          // reliable updates performed (mixed)
    int* flag;        // per-iteration scratch flag (mixed: update requested)
};

__device__ Smem carve(int nrhs)
{
    extern __shared__ double sm[];
    Smem s;
    s.scratch = sm;
    s.rr = sm + 64;
    s.bb = s.rr + nrhs;
    s.cf = s.bb + nrhs;
    s.al = s.cf + nrhs;
    s.aux = s.al + nrhs;
    s.rru = s.aux + nrhs;
    int* ib = reinterpret_cast<int*>(s.rru + nrhs);
    s.state = ib;
    s.iters = ib + nrhs;
    s.act = s.iters + nrhs;
    s.ru = s.act + nrhs;
    s.flag = s.ru + nrhs;
    return s;
}

// Compact {j : pred(j)} into act in increasing j. Same result in every block.
template <typename P>
__device__ int compact(int nrhs, int* act, double* scratch, P pred)
{
    int* cnt = reinterpret_cast<int*>(scratch);  // 32 ints
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int base = 0;
    for (int j0 = 0; j0 < nrhs; j0 += blockDim.x)
    {
        const int j = j0 + threadIdx.x;
        const int f = (j < nrhs && pred(j)) ? 1 : 0;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        const int pre = __popc(m & ((1u << lane) - 1u));
        __syncthreads();
        if (lane == 0)
            cnt[w] = __popc(m);
        __syncthreads();
        int off = 0, total = 0;
        for (int k = 0; k < nw; ++k)
        {
            if (k < w)
                off += cnt[k];
            total += cnt[k];
        }
        if (f)
            act[base + off + pre] = j;
        base += total;
    }
    __syncthreads();
    return base;
}

// Sum of the `slot` partials of every listed right-hand side into out[j].
__device__ void reduce_listed(const SolveDesc& d, const int* act, int nact, int slot, double* out)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = w; k < nact; k += nw)
    {
        const int j = act[k];
        double v = 0.0;
        for (int c = lane; c < d.nch; c += 32)
            v += __ldcg(&d.part[(long(j) * d.nch + c) * 2 + slot]);
        v = warp_sum(v);
        if (lane == 0)
            out[j] = v;
    }
    __syncthreads();
}

// Visit every site of every listed right-hand side; f(j, i) returns two
// partial-sum contributions, stored per unit when `keep` is set.
template <typename F>
__device__ void sweep(const SolveDesc& d, const int* act, int nact, double* scratch, bool keep,
                      F f)
{
    const int nunits = nact * d.nch;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x)
    {
        const int k = u / d.nch, c = u - k * d.nch, j = act[k];
        const int beg = c * d.ch;
        const int end = min(beg + d.ch, d.L.nsite);
        const long uo = long(d.rhs_conf[j]) * d.usz;  // this unit's link offset
        double a0 = 0.0, a1 = 0.0;
        for (int i = beg + threadIdx.x; i < end; i += blockDim.x)
        {
            const double2 v = f(j, i, uo);
            a0 += v.x;
            a1 += v.y;
        }
        if (keep)
        {
            a0 = block_sum(a0, scratch);
            a1 = block_sum(a1, scratch);
            if (threadIdx.x == 0)
            {
                d.part[(long(j) * d.nch + c) * 2] = a0;
                d.part[(long(j) * d.nch + c) * 2 + 1] = a1;
            }
        }
    }
}

template <typename R>
__device__ __forceinline__ Spinor<R> op_site(const SolveDesc& d, bool dag,
                                             const cplx<R>* __restrict__ in,
                                             const cplx<R>* __restrict__ U, int i)
{
    int s, t, x;
    site_coords(d.L, i, s, t, x);
    return dag ? dirac_site<true, R>(in, U, d.L, s, t, x)
               : dirac_site<false, R>(in, U, d.L, s, t, x);
}



__device__ __forceinline__ Spinor<float> to32(const Spinor<double>& v)
{
    return {make_float2(float(v.s0.x), float(v.s0.y)), make_float2(float(v.s1.x), float(v.s1.y))};
}
__device__ __forceinline__ Spinor<double> to64(const Spinor<float>& v)
{
    return {make_double2(v.s0.x, v.s0.y), make_double2(v.s1.x, v.s1.y)};
}
__device__ __forceinline__ Spinor<double> axpy(double a, const Spinor<double>& x,
                                               const Spinor<double>& y)
{
    return {a * x.s0 + y.s0, a * x.s1 + y.s1};
}
__device__ __forceinline__ Spinor<float> axpy(float a, const Spinor<float>& x,
                                              const Spinor<float>& y)
{
    return {a * x.s0 + y.s0, a * x.s1 + y.s1};
}

// r + beta p_old formed on the fly: the fused direction update.
template <typename R>
struct DirLd
{
    const cplx<R>* __restrict__ r;
    const cplx<R>* __restrict__ p;
    R beta;
    __device__ __forceinline__ Spinor<R> sp(long site) const
    {
        const Spinor<R> a = ld_spinor(r, site);
        const Spinor<R> b = ld_spinor(p, site);
        return {a.s0 + beta * b.s0, a.s1 + beta * b.s1};
    }
    __device__ __forceinline__ cplx<R> c(long idx) const { return r[idx] + beta * p[idx]; }
};

template <typename R, typename Ld>
__device__ __forceinline__ Spinor<R> op_site_ld(const SolveDesc& d, bool dag, const Ld& in,
                                                const cplx<R>* __restrict__ U, int i)
{
    int s, t, x;
    site_coords(d.L, i, s, t, x);
    return dag ? dirac_site_ld<true, R>(in, U, d.L, s, t, x)
               : dirac_site_ld<false, R>(in, U, d.L, s, t, x);
}

__device__ void write_outputs(const SolveDesc& d, const Smem& s)
{
    if (blockIdx.x != 0)
        return;
    for (int j = threadIdx.x; j < d.nrhs; j += blockDim.x)
    {
        d.out_iters[j] = s.iters[j];
        d.out_status[j] = s.state[j] == RHS_ACTIVE ? DWF_NOT_CONVERGED : s.state[j];
        d.out_relres[j] = s.bb[j] > 0.0 ? sqrt(s.rr[j] / s.bb[j]) : 0.0;
        d.out_ru[j] = s.ru[j];
    }
}

// Initial residual: r = b - A x (guess) or r = b (x = 0 set by the host).
// Leaves |b|^2 in bb and |r|^2 in rr. Returns false on a barrier error.
__device__ bool init_residual(const SolveDesc& d, const Smem& s, int nact, bool mixed)
{
    const long fs = d.fsz;
    const bool dag1 = d.dag_first != 0;
    if (d.has_guess)
    {
        sweep(d, s.act, nact, s.scratch, false, [&](int j, int i, long uo) {
            const Spinor<double> v = op_site<double>(d, dag1, d.x + j * fs, d.U64 + uo, i);
            st_spinor(d.t + j * fs, i, v);
            return make_double2(0.0, 0.0);
        });
        if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
            return false;
    }
    sweep(d, s.act, nact, s.scratch, true, [&](int j, int i, long uo) {
        const Spinor<double> b = ld_spinor(d.b + j * fs, i);
        Spinor<double> r = b;
        if (d.has_guess)
        {
            const Spinor<double> a =
                op_site<double>(d, !dag1, d.t + j * fs, d.U64 + uo, i);
            r = {b.s0 - a.s0, b.s1 - a.s1};
        }
        st_spinor(d.r + j * fs, i, r);
        if (mixed)
        {
            const Spinor<float> r32 = to32(r);
            st_spinor(d.r32 + j * fs, i, r32);
            st_spinor(d.p32 + j * fs, i, r32);
            st_spinor(d.e32 + j * fs, i, Spinor<float>{make_float2(0.f, 0.f), make_float2(0.f, 0.f)});
        }
        else
        {
            st_spinor(d.p + j * fs, i, r);
        }
        return make_double2(spinor_norm2(b), spinor_norm2(r));
    });
    if (!grid_sync(d.bar, d.expected_blocks, d.timeout_ns))
        return false;
    reduce_listed(d, s.act, nact, 0, s.bb);
    reduce_listed(d, s.act, nact, 1, s.rr);
    return true;
}

// Initial convergence test (cg_solver.hpp:30-38; Eigen rule: |r|^2 < tol^2 |b|^2).
__device__ bool converged_now(const SolveDesc& d, double rr, double bb)
{
    if (d.eigen_rule)
        return rr < fmax(d.rtol * d.rtol * bb, 2.2250738585072014e-308);
    return sqrt(rr) / sqrt(bb) <= d.rtol;
}

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
        const int nru = compact(d.nrhs, s.act, s.scratch, [&](int j) {
            return s.state[j] == RHS_ACTIVE && (s.flag[j] & 1);
        });
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
