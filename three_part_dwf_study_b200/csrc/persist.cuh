// Building blocks of the persistent solver kernels: per-right-hand-side state
// in shared memory, active-list compaction, unit sweeps with per-unit partial
// sums, deterministic per-right-hand-side reductions and the common
// initial-residual / output steps.
#pragma once

#include "solver.cuh"

#ifndef DWFB_SWEEP_UNROLL
#define DWFB_SWEEP_UNROLL 1  // sites per thread whose loads the sweep loop may overlap
#endif

namespace dwfb {
namespace persist {

constexpr int kSweepUnroll = DWFB_SWEEP_UNROLL;

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

__device__ inline Smem carve(int nrhs)
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
__device__ inline void reduce_listed(const SolveDesc& d, const int* act, int nact, int slot, double* out)
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

// Visit sites [0, nsite) of every listed right-hand side in units of `ch`
// sites (nch units per right-hand side); f(j, i, uo) returns two partial-sum
// contributions, stored per unit when `keep` is set (uo: the unit's link offset).
template <typename F>
__device__ void sweep_sites(const SolveDesc& d, const int* act, int nact, int nsite, int nch,
                            int ch, double* scratch, bool keep, F f)
{
    const int nunits = nact * nch;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x)
    {
        const int k = u / nch, c = u - k * nch, j = act[k];
        const int beg = c * ch;
        const int end = min(beg + ch, nsite);
        const long uo = long(d.rhs_conf[j]) * d.usz;  // this unit's link offset
        double a0 = 0.0, a1 = 0.0;
#pragma unroll kSweepUnroll
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
                d.part[(long(j) * nch + c) * 2] = a0;
                d.part[(long(j) * nch + c) * 2 + 1] = a1;
            }
        }
    }
}

// The full-lattice sweep (nsite = Ls*V, the launch's chunking).
template <typename F>
__device__ void sweep(const SolveDesc& d, const int* act, int nact, double* scratch, bool keep,
                      F f)
{
    sweep_sites(d, act, nact, d.L.nsite, d.nch, d.ch, scratch, keep, f);
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

__device__ inline void write_outputs(const SolveDesc& d, const Smem& s)
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
__device__ inline bool init_residual(const SolveDesc& d, const Smem& s, int nact, bool mixed)
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
__device__ inline bool converged_now(const SolveDesc& d, double rr, double bb)
{
    if (d.eigen_rule)
        return rr < fmax(d.rtol * d.rtol * bb, 2.2250738585072014e-308);
    return sqrt(rr) / sqrt(bb) <= d.rtol;
}

}  // namespace persist
}  // namespace dwfb
