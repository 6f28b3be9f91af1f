// Non-persistent kernels: link phases, operator application, residual norms.
#pragma once

#include "dirac.cuh"

namespace dwfb {

// theta[c][mu][t][x] -> U64 = (cos, sin), U32 = rounded copy.
__global__ void links_kernel(const double* __restrict__ theta, long n, double2* __restrict__ U64,
                             float2* __restrict__ U32);

// out[j] = D or D^dag (in[j]) on configuration conf[j] (conf may be null -> conf0).
template <bool DAG, typename R>
__global__ void dirac_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                             long fsz, const cplx<R>* __restrict__ U, long usz,
                             const int* __restrict__ conf, int conf0);

// Same operator, one thread per 5-D site with the x neighbours exchanged by
// warp shuffles (needs Nx % 32 == 0).
template <bool DAG, typename R>
__global__ void dirac_warp_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                  long fsz, const cplx<R>* __restrict__ U, long usz,
                                  const int* __restrict__ conf, int conf0);

// Same operator, one thread per 4-D site sweeping s like dirac_col_kernel,
// with the x neighbours and the backward x link exchanged by warp shuffles
// (Nx % 32 == 0; the two edge lanes load theirs), slice s+1's spinor loads
// issued before slice s is computed and slice s+DWFB_COLX_PREFETCH prefetched
// into L1 (grid: Nx/32 x ceil(Nt/8) x nrhs, 256 threads, one t row per warp;
// launched with the largest-L1 shared-memory split preferred).
template <bool DAG, typename R>
__global__ void dirac_colx_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                  long fsz, const cplx<R>* __restrict__ U, long usz,
                                  const int* __restrict__ conf, int conf0);

// Same operator over a block-shared ring of kRingSlots slices in shared
// memory, filled by 1-D bulk copies (cp.async.bulk, mbarrier completion): a
// block of 8 warps covers 32 x by kRingT t rows and sweeps s; warp 0 copies
// each slice's kRingRows x kRingWidth sites (the tile and its halo) kRingSlots
// slices ahead, every neighbour is read from shared memory, and a block
// barrier per slice frees the slot for the next copy (Nx % 32 == 0,
// Nt % kRingT == 0; grid Nx/32 x Nt/kRingT x nrhs, 256 threads, dynamic
// shared memory tile_smem_bytes). Warp w copies its own t row (warps 0 and
// 7 also the halo rows), signals an mbarrier of its own per slot, and refills
// a slot once all eight warps have arrived on the slot's release barrier. A
// wait longer than limit_ns sets *err to DWF_TIMEOUT and ends the warp once
// its own copies have landed.
#ifndef DWFB_RING_SLOTS
#define DWFB_RING_SLOTS 4
#endif
constexpr int kRingT = 8, kRingRows = kRingT + 2, kRingWidth = 34, kRingSlots = DWFB_RING_SLOTS;
#ifndef DWFB_TILE_MINB64
#define DWFB_TILE_MINB64 4  // resident blocks per SM asked of the FP64 build
#endif
#ifndef DWFB_TILE_MINB32
#define DWFB_TILE_MINB32 4
#endif
__host__ __device__ constexpr size_t tile_smem_bytes(size_t site_bytes)
{
    return size_t(kRingSlots) * kRingRows * kRingWidth * site_bytes + 8 * kRingSlots * (kRingT + 1);
}
template <bool DAG, typename R>
__global__ void dirac_tile_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                  long fsz, const cplx<R>* __restrict__ U, long usz,
                                  const int* __restrict__ conf, int conf0, int* err,
                                  unsigned long long limit_ns);

// Wilson only (Ls = 1, no fifth dimension; Nx % 32 == 0, Nt % RT == 0): a
// warp covers 32 consecutive x of RT consecutive rows, each thread loading
// its column's rows t0-1 .. t0+RT into registers up front (RT + 2 spinor loads
// for RT sites), the x neighbours and backward x link by shuffle, the two
// edge lanes loading theirs (grid: Nx/32 x ceil(Nt/(RT by)) x nrhs, block
// (32, by)).
constexpr int kWilsonRows = 4;
template <bool DAG, typename R, int RT>
__global__ void wilson_rows_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                   long fsz, const cplx<R>* __restrict__ U, long usz,
                                   const int* __restrict__ conf, int conf0);

// Same operator, one thread per 4-D site sweeping the fifth dimension
// (grid: ceil(Nx/32) x ceil(Nt/8) x nrhs, 256 threads).
template <bool DAG, typename R>
__global__ void dirac_col_kernel(Lat L, const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                 long fsz, const cplx<R>* __restrict__ U, long usz,
                                 const int* __restrict__ conf, int conf0);

// Same operator, one thread per (s, x) sweeping a chunk of tc rows in t,
// RPS rows per step, through a ring of (NPG + 1) * RPS shared-memory row
// slots filled by cp.async (grid: Nx/(32 G) x ceil(Nt/tc) x nrhs, block
// (32, Ls, G), Nx % 32 == 0, 32 Ls G <= 512, dynamic shared memory
// (NPG + 1) * RPS * sweep_slot_bytes).
constexpr int kSweepRows64 = 1, kSweepGroups64 = 4;   // two FP64 rows per step need one block per SM: slower
constexpr int kSweepRows32 = 2, kSweepGroups32 = 3;
constexpr int sweep_ring_rows(int npg, int rps) { return (npg + 1) * rps; }

// One ring slot: spinors [Ls][32 G + 2] (halo column each side), t links
// [32 G], x links [32 G + 1] (left halo first), rounded up to 16 bytes.
__host__ __device__ constexpr size_t sweep_slot_bytes(int Ls, int G, size_t csize)
{
    return ((size_t(2) * Ls * (32 * G + 2) + 64 * G + 1) * csize + 15) / 16 * 16;
}

template <bool DAG, typename R, int NPG, int RPS>
__global__ void dirac_sweep_kernel(Lat L, const cplx<R>* __restrict__ in,
                                   cplx<R>* __restrict__ out, long fsz,
                                   const cplx<R>* __restrict__ U, long usz,
                                   const int* __restrict__ conf, int conf0, int tc);

// Per-(rhs, chunk) partials of |b - D2 t|^2 and |b|^2 (true residual of A x = b
// after t = D1 x).
template <bool DAG>
__global__ void residual_partials_kernel(Lat L, const double2* __restrict__ t,
                                         const double2* __restrict__ b, long fsz,
                                         const double2* __restrict__ U, long usz,
                                         const int* __restrict__ conf, int nch, int ch,
                                         double* __restrict__ part);

// out[j] = sqrt(sum part[j][.][0] / sum part[j][.][1]), one warp per rhs.
__global__ void residual_finish_kernel(const double* __restrict__ part, int nrhs, int nch,
                                       double* __restrict__ out);

// Grid-barrier self test (see dwf_barrier_selftest).
__global__ void barrier_probe_kernel(GridBar* bar, unsigned expected, unsigned long long timeout_ns,
                                     int rounds);

}  // namespace dwfb
