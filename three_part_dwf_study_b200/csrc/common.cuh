// Shared device helpers: complex arithmetic on double2/float2, spinor loads,
// a bounded grid-wide barrier for persistent cooperative kernels, and
// deterministic block reductions.
#pragma once

#include <cuda_runtime.h>
#include <cuda/atomic>
#include <cstdint>

#include "../../include/dwf_b200.h"

namespace dwfb {

// ---------------------------------------------------------------------------
// complex types
// ---------------------------------------------------------------------------
template <typename R> struct CT;
template <> struct CT<double> { using c = double2; };
template <> struct CT<float> { using c = float2; };
template <typename R> using cplx = typename CT<R>::c;

__host__ __device__ __forceinline__ double2 mkc(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 mkc(float a, float b) { return make_float2(a, b); }

#define DWFB_CPLX_OPS(T, R)                                                                      \
    __device__ __forceinline__ T operator+(T a, T b) { return mkc(a.x + b.x, a.y + b.y); }     \
    __device__ __forceinline__ T operator-(T a, T b) { return mkc(a.x - b.x, a.y - b.y); }     \
    __device__ __forceinline__ T operator-(T a) { return mkc(-a.x, -a.y); }                    \
    __device__ __forceinline__ T operator*(R k, T a) { return mkc(k * a.x, k * a.y); }         \
    __device__ __forceinline__ T& operator+=(T& a, T b) { a.x += b.x; a.y += b.y; return a; }  \
    __device__ __forceinline__ T cmul(T a, T b)                                                \
    {                                                                                          \
        return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);                              \
    }                                                                                          \
    /* conj(a) * b */                                                                          \
    __device__ __forceinline__ T cmulc(T a, T b)                                               \
    {                                                                                          \
        return mkc(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);                              \
    }                                                                                          \
    /* i * a */                                                                                \
    __device__ __forceinline__ T itimes(T a) { return mkc(-a.y, a.x); }                        \
    __device__ __forceinline__ R norm2(T a) { return a.x * a.x + a.y * a.y; }

DWFB_CPLX_OPS(double2, double)
DWFB_CPLX_OPS(float2, float)
#undef DWFB_CPLX_OPS

// A lattice site carries a 2-component spinor: two complex numbers, stored
// consecutively (spin fastest), so one site is 32 B in FP64 and 16 B in FP32.
template <typename R>
struct Spinor
{
    cplx<R> s0, s1;
};

__device__ __forceinline__ Spinor<double> ld_spinor(const double2* __restrict__ f, long site)
{
    const double2* p = f + 2 * site;
    return {p[0], p[1]};
}
__device__ __forceinline__ Spinor<float> ld_spinor(const float2* __restrict__ f, long site)
{
    const float4 v = reinterpret_cast<const float4*>(f)[site];
    return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ void st_spinor(double2* __restrict__ f, long site, Spinor<double> v)
{
    double2* p = f + 2 * site;
    p[0] = v.s0;
    p[1] = v.s1;
}
__device__ __forceinline__ void st_spinor(float2* __restrict__ f, long site, Spinor<float> v)
{
    reinterpret_cast<float4*>(f)[site] = make_float4(v.s0.x, v.s0.y, v.s1.x, v.s1.y);
}

template <typename R>
__device__ __forceinline__ double spinor_norm2(const Spinor<R>& v)
{
    return double(v.s0.x) * v.s0.x + double(v.s0.y) * v.s0.y + double(v.s1.x) * v.s1.x +
           double(v.s1.y) * v.s1.y;
}

// ---------------------------------------------------------------------------
// lattice geometry shared by every kernel
// ---------------------------------------------------------------------------
struct Lat
{
    int Nt, Nx, Ls;  // Ls = 1 for Wilson
    int V;           // Nt * Nx
    int nsite;       // Ls * V (2-spinor sites per right-hand side)
    double diag;     // 3 - M5 (domain wall) or 2 + m0 (Wilson)
    double mf;       // domain-wall quark mass (unused for Wilson)
    double bct, bcx; // fermion boundary signs in t and x
    int fifth;       // 1: domain-wall fifth-dimension hop present
};

// ---------------------------------------------------------------------------
// bounded grid barrier (persistent cooperative kernels)
// ---------------------------------------------------------------------------
struct GridBar
{
    unsigned int count;
    unsigned int gen;
    int err;      // first error code raised by any block (0 = none)
    int pad;
};

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// All blocks of a cooperative launch call this in the same order. Returns
// false (in every thread of the block) once any block has recorded an error,
// including a wait that ran past `timeout_ns`; the caller then leaves its loop.
// `expected` is the number of arriving blocks (gridDim.x in normal use).
__device__ __forceinline__ bool grid_sync(GridBar* bar, unsigned expected,
                                          unsigned long long timeout_ns)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(bar->gen);
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(bar->count);
        cuda::atomic_ref<int, cuda::thread_scope_device> err(bar->err);
        const unsigned g = gen.load(cuda::memory_order_relaxed);
        const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        int good = 1;
        if (arrived == expected - 1)
        {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        }
        else
        {
            const unsigned long long t0 = globaltimer_ns();
            while (gen.load(cuda::memory_order_acquire) == g)
            {
                if (err.load(cuda::memory_order_relaxed) != 0)
                {
                    good = 0;
                    break;
                }
                if (globaltimer_ns() - t0 > timeout_ns)
                {
                    int zero = 0;
                    err.compare_exchange_strong(zero, DWF_TIMEOUT, cuda::memory_order_relaxed);
                    good = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        cuda::atomic_thread_fence(cuda::memory_order_acq_rel, cuda::thread_scope_device);
        ok = good && err.load(cuda::memory_order_relaxed) == 0;
    }
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ void raise_error(GridBar* bar, int code)
{
    cuda::atomic_ref<int, cuda::thread_scope_device> err(bar->err);
    int zero = 0;
    err.compare_exchange_strong(zero, code, cuda::memory_order_relaxed);
}

// ---------------------------------------------------------------------------
// deterministic reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum in a fixed order; the result is valid in every thread.
// `scratch` holds at least 32 doubles; blockDim.x is a multiple of 32.
__device__ __forceinline__ double block_sum(double v, double* scratch)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0)
        scratch[w] = v;
    __syncthreads();
    double t = (lane < nw) ? scratch[lane] : 0.0;
    if (w == 0)
        t = warp_sum(t);
    __syncthreads();
    if (threadIdx.x == 0)
        scratch[0] = t;
    __syncthreads();
    const double r = scratch[0];
    __syncthreads();
    return r;
}

}  // namespace dwfb
