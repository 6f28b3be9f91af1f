// Analyzer measurements: boundary sources, batched propagator solves and the
// meson contractions (domain_wall/include/correlator.hpp:27-310,
// wilson/include/correlator.hpp:10-40), for many configurations at once.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "context.cuh"
#include "kernels.cuh"

using namespace dwfb;

#define CK(call)                                                                        \
    do                                                                                  \
    {                                                                                   \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ctx_fail(c, DWF_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

namespace dwfb {

// Source kinds, per configuration in this order:
//   point: n_point times x 2 spins, wall: n_wall times x 2 spins, noise: n_noise.
// P_L = diag(0, 1), P_R = diag(1, 0): column b = 1 of P_L sits on spin 1 at
// s = 0, column b = 0 of P_R on spin 0 at s = Ls-1 (correlator.hpp:133-138,
// :201-211); a noise vector eta contributes P_L eta at s = 0 and P_R eta at
// s = Ls-1 (:60-75).
struct SrcDesc
{
    Lat L;
    int R;  // right-hand sides per configuration
    int n_point, n_wall, n_noise;
    int ls_src;         // domain wall: 1 (boundary sources); Wilson: 0 (plain point source)
    int src_x;          // point-source x (domain wall: 0)
    int wil_t;          // Wilson point-source t
    const signed char* z4;  // [nconf][n_noise][Nt][Nx][2]
};

__device__ __forceinline__ int src_time(int k, int n, int Nt) { return (k * Nt) / n; }

__global__ void sources_kernel(SrcDesc d, long nrhs, double2* __restrict__ src)
{
    const long fsz = 2L * d.L.nsite;
    const long total = nrhs * fsz;
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < total;
         idx += long(gridDim.x) * blockDim.x)
    {
        const long j = idx / fsz;
        const int e = int(idx - j * fsz);  // complex index within the field
        const int a = e & 1;
        const int site = e >> 1;
        const int s = site / d.L.V;
        const int r = site - s * d.L.V;
        const int t = r / d.L.Nx, x = r - t * d.L.Nx;
        const int conf = int(j / d.R), k = int(j - long(conf) * d.R);
        double2 v = make_double2(0.0, 0.0);
        if (!d.ls_src)
        {
            // Wilson: source[site_index(src_t, src_x, b)] = 1 (wilson/include/correlator.hpp:17-18)
            if (t == d.wil_t && x == d.src_x && a == k)
                v.x = 1.0;
        }
        else if (k < 2 * d.n_point)
        {
            const int ts = src_time(k >> 1, d.n_point, d.L.Nt), b = k & 1;
            if (t == ts && x == d.src_x && a == b && ((b == 1 && s == 0) || (b == 0 && s == d.L.Ls - 1)))
                v.x = 1.0;
        }
        else if (k < 2 * d.n_point + 2 * d.n_wall)
        {
            const int kk = k - 2 * d.n_point;
            const int ts = src_time(kk >> 1, d.n_wall, d.L.Nt), b = kk & 1;
            if (t == ts && a == b && ((b == 1 && s == 0) || (b == 0 && s == d.L.Ls - 1)))
                v.x = 1.0;
        }
        else
        {
            const int nz = k - 2 * d.n_point - 2 * d.n_wall;
            const long zi = ((long(conf) * d.n_noise + nz) * d.L.V + r) * 2 + a;
            const int dig = d.z4[zi];
            // phases {1, i, -1, -i} (correlator.hpp:37-39)
            const double2 ph = make_double2(dig == 0 ? 1.0 : (dig == 2 ? -1.0 : 0.0),
                                            dig == 1 ? 1.0 : (dig == 3 ? -1.0 : 0.0));
            if ((a == 1 && s == 0) || (a == 0 && s == d.L.Ls - 1))
                v = ph;
        }
        src[idx] = v;
    }
}

// One block per (right-hand side, t): sums over x of
//   [0] |q|^2, [1] Re(psi(Ls/2)^dag q), [2+n] cos(2 pi n x / Nx) |q|^2,
// with q = P_L psi(s=0) + P_R psi(s=Ls-1) = (psi_0(Ls-1), psi_1(0))
// (correlator.hpp:149-174, :258-301). Wilson (ls_src = 0): [0] = sum_x sum_a
// |psi_a(t,x)|^2 (wilson/include/correlator.hpp:32-39). The per-x values are
// staged in shared memory (2*Nx doubles); each output is one warp's fixed-order
// sum over x.
__global__ void contract_kernel(Lat L, int ls_src, int nmom, const double2* __restrict__ psi,
                                double* __restrict__ red)
{
    extern __shared__ double sx[];  // [Nx] |q|^2, [Nx] J5
    const long j = blockIdx.y;
    const int t = blockIdx.x;
    const int K = 2 + nmom;
    const double2* P = psi + j * 2L * L.nsite;
    double* qq = sx;
    double* j5 = sx + L.Nx;
    for (int x = threadIdx.x; x < L.Nx; x += blockDim.x)
    {
        const int site = t * L.Nx + x;
        if (!ls_src)
        {
            qq[x] = spinor_norm2(ld_spinor(P, site));
            j5[x] = 0.0;
            continue;
        }
        const double2 q0 = P[2 * (long(L.Ls - 1) * L.V + site)];
        const double2 q1 = P[2 * long(site) + 1];
        const Spinor<double> mid = ld_spinor(P, long(L.Ls / 2) * L.V + site);
        qq[x] = norm2(q0) + norm2(q1);
        j5[x] = mid.s0.x * q0.x + mid.s0.y * q0.y + mid.s1.x * q1.x + mid.s1.y * q1.y;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = w; k < K; k += nw)
    {
        double acc = 0.0;
        for (int x = lane; x < L.Nx; x += 32)
        {
            if (k == 0)
                acc += qq[x];
            else if (k == 1)
                acc += j5[x];
            else
                acc += cos(2.0 * 3.141592653589793238462643383279502884 * (k - 2) / L.Nx * x) * qq[x];
        }
        acc = warp_sum(acc);
        if (lane == 0)
            red[(j * L.Nt + t) * K + k] = acc;
    }
}

// loop(conf, t, x) = (1/n_noise) sum_noise eta^dag gamma5 q,  gamma5 = diag(1, -1)
// (correlator.hpp:83-107), summed over the noise vectors in order.
__global__ void loop_kernel(Lat L, int R, int first_noise, int n_noise, long nconf,
                            const signed char* __restrict__ z4, const double2* __restrict__ psi,
                            double2* __restrict__ loop)
{
    const long total = nconf * L.V;
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < total;
         idx += long(gridDim.x) * blockDim.x)
    {
        const long conf = idx / L.V;
        const int site = int(idx - conf * L.V);
        double2 acc = make_double2(0.0, 0.0);
        for (int nz = 0; nz < n_noise; ++nz)
        {
            const long j = conf * R + first_noise + nz;
            const double2* P = psi + j * 2L * L.nsite;
            const double2 q0 = P[2 * (long(L.Ls - 1) * L.V + site)];
            const double2 q1 = P[2 * long(site) + 1];
            const long zi = ((conf * n_noise + nz) * L.V + site) * 2;
            double2 e[2];
            for (int a = 0; a < 2; ++a)
            {
                const int dig = z4[zi + a];
                e[a] = make_double2(dig == 0 ? 1.0 : (dig == 2 ? -1.0 : 0.0),
                                    dig == 1 ? 1.0 : (dig == 3 ? -1.0 : 0.0));
            }
            acc += cmulc(e[0], q0);
            acc += -cmulc(e[1], q1);
        }
        loop[idx] = make_double2(acc.x / n_noise, acc.y / n_noise);
    }
}

}  // namespace dwfb

namespace {

// Grow-only device buffer of the context (freed by dwf_ctx_destroy).
template <typename T>
int reserve(dwf_ctx* c, T*& p, size_t& cap, size_t n)
{
    n = std::max<size_t>(n, 1);
    if (p && n <= cap)
        return DWF_OK;
    CK(cudaStreamSynchronize(c->stream));
    if (p)
        cudaFree(p);
    p = nullptr;
    cap = 0;
    CK(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)));
    cap = n;
    return DWF_OK;
}

}  // namespace

extern "C" {

int dwf_measure(dwf_ctx* c, const dwf_measure_params* mp, int nconf, const double* thetas,
                const signed char* z4, double* cpp, double* cj5, double* loop, double* mom_cpp,
                dwf_solve_info* info)
{
    if (!c || !mp || !thetas || nconf < 1 || c->kind != 0)
        return DWF_BAD_ARG;
    if (mp->n_point_times < 0 || mp->n_wall_times < 0 || mp->n_noise < 0 ||
        mp->max_momentum < 0 || mp->max_momentum > c->L.Nx / 2)
        return ctx_fail(c, DWF_BAD_ARG, "analysis.max_momentum is outside 0..Nx/2");
    if (mp->n_noise > 0 && !z4)
        return ctx_fail(c, DWF_BAD_ARG, "measure: z4 digits required for noise sources");
    const int R = 2 * mp->n_point_times + 2 * mp->n_wall_times + mp->n_noise;
    if (R < 1)
        return ctx_fail(c, DWF_BAD_ARG, "measure: no sources");
    CK(cudaSetDevice(c->device));
    int st = set_gauge(c, nconf, thetas, cudaMemcpyHostToDevice);
    if (st)
        return st;
    const long nrhs = long(nconf) * R;
    const long fs = c->fsz();
    const int nmom = mp->n_point_times > 0 ? mp->max_momentum + 1 : 0;
    const int K = 2 + nmom;
    // sources and solutions in the solver workspace's staging fields, the rest
    // in the context's measurement buffers: no allocation once they have grown
    if ((st = ensure_workspace(c, int(nrhs))) ||
        (st = reserve(c, c->m_red, c->m_red_cap, size_t(nrhs) * c->L.Nt * K)) ||
        (st = reserve(c, c->m_loop, c->m_loop_cap, size_t(nconf) * c->L.V)) ||
        (st = reserve(c, c->m_z4, c->m_z4_cap, size_t(nconf) * mp->n_noise * c->L.V * 2)))
        return st;
    struct
    {
        double2* src;
        double2* x;
        double* red;
        signed char* z4;
        double2* loop;
    } B{c->w_src, c->w_x, c->m_red, c->m_z4, c->m_loop};
    if (mp->n_noise > 0 &&
        cudaMemcpyAsync(B.z4, z4, long(nconf) * mp->n_noise * c->L.V * 2, cudaMemcpyHostToDevice,
                        c->stream) != cudaSuccess)
        return ctx_fail(c, DWF_CUDA_ERROR, "measure: z4 upload failed");
    SrcDesc sd{};
    sd.L = c->L;
    sd.R = R;
    sd.n_point = mp->n_point_times;
    sd.n_wall = mp->n_wall_times;
    sd.n_noise = mp->n_noise;
    sd.ls_src = 1;
    sd.src_x = 0;
    sd.z4 = B.z4;
    sources_kernel<<<std::max(1, 8 * c->nsm), 256, 0, c->stream>>>(sd, nrhs, B.src);
    c->launches += 1;
    std::vector<int> conf(nrhs);
    for (long j = 0; j < nrhs; ++j)
        conf[j] = int(j / R);
    std::vector<dwf_solve_info> inf(nrhs);
    st = propagators(c, int(nrhs), conf.data(), B.src, B.x, mp->rtol, mp->maxiter, mp->solver,
                     inf.data());
    if (st)
        return st;
    for (long j = 0; j < nrhs; j += 65535)
    {
        const int n = int(std::min<long>(65535, nrhs - j));
        contract_kernel<<<dim3(c->L.Nt, n), 128, 2 * c->L.Nx * sizeof(double), c->stream>>>(
            c->L, 1, nmom, B.x + j * fs, B.red + j * c->L.Nt * K);
        c->launches += 1;
    }
    if (mp->n_noise > 0)
    {
        loop_kernel<<<std::max(1, 4 * c->nsm), 256, 0, c->stream>>>(
            c->L, R, 2 * mp->n_point_times + 2 * mp->n_wall_times, mp->n_noise, nconf, B.z4, B.x,
            B.loop);
        c->launches += 1;
    }
    if (cudaGetLastError() != cudaSuccess)
        return ctx_fail(c, DWF_CUDA_ERROR, "measure: kernel launch failed");
    std::vector<double> red(nrhs * c->L.Nt * K);
    std::vector<double> lp(mp->n_noise > 0 ? 2L * nconf * c->L.V : 0);
    cudaMemcpyAsync(red.data(), B.red, red.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (!lp.empty())
        cudaMemcpyAsync(lp.data(), B.loop, lp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess)
        return ctx_fail(c, DWF_CUDA_ERROR, "measure: copy-back failed");

    const int Nt = c->L.Nt;
    auto R_at = [&](long j, int t, int k) { return red[(j * Nt + t) * K + k]; };
    for (int cf = 0; cf < nconf; ++cf)
    {
        // C_PP, C_J5 from the wall sources, averaged over source times
        // (compute_CPP_CJ5, correlator.hpp:243-310)
        if (cpp || cj5)
            for (int t = 0; t < Nt; ++t)
            {
                if (cpp)
                    cpp[long(cf) * Nt + t] = 0.0;
                if (cj5)
                    cj5[long(cf) * Nt + t] = 0.0;
            }
        for (int kt = 0; kt < mp->n_wall_times; ++kt)
        {
            const int ts = (kt * Nt) / mp->n_wall_times;
            for (int t = 0; t < Nt; ++t)
            {
                const int dt = (t - ts + Nt) % Nt;
                for (int b = 0; b < 2; ++b)
                {
                    const long j = long(cf) * R + 2 * mp->n_point_times + 2 * kt + b;
                    if (cpp)
                        cpp[long(cf) * Nt + dt] += R_at(j, t, 0);
                    if (cj5)
                        cj5[long(cf) * Nt + dt] += R_at(j, t, 1);
                }
            }
        }
        if (mp->n_wall_times > 0)
            for (int t = 0; t < Nt; ++t)
            {
                if (cpp)
                    cpp[long(cf) * Nt + t] /= double(mp->n_wall_times);
                if (cj5)
                    cj5[long(cf) * Nt + t] /= double(mp->n_wall_times);
            }
        // momentum-projected C_PP from the point sources (compute_momentum_CPP, :111-181)
        if (mom_cpp && nmom > 0)
        {
            double* M = mom_cpp + long(cf) * nmom * Nt;
            std::fill(M, M + long(nmom) * Nt, 0.0);
            for (int kt = 0; kt < mp->n_point_times; ++kt)
            {
                const int ts = (kt * Nt) / mp->n_point_times;
                for (int t = 0; t < Nt; ++t)
                {
                    const int dt = (t - ts + Nt) % Nt;
                    for (int n = 0; n < nmom; ++n)
                        for (int b = 0; b < 2; ++b)
                            M[n * Nt + dt] += R_at(long(cf) * R + 2 * kt + b, t, 2 + n);
                }
            }
            for (long i = 0; i < long(nmom) * Nt; ++i)
                M[i] /= double(mp->n_point_times);
        }
        if (loop && mp->n_noise > 0)
            std::copy(lp.begin() + 2L * cf * c->L.V, lp.begin() + 2L * (cf + 1) * c->L.V,
                      loop + 2L * cf * c->L.V);
    }
    if (info)
        std::copy(inf.begin(), inf.end(), info);
    return DWF_OK;
}

// pseudoscalar_correlator (wilson/include/correlator.hpp:10-40) for nconf
// configurations: two point sources at (src_t, src_x), CGNR solves with the
// 20 tol check of solve_CGNR, C(t) = sum_{x, a, b} |S(t, x, a; b)|^2.
int wil_pseudoscalar_correlator(dwf_ctx* c, int nconf, const double* thetas, int src_t, int src_x,
                                double tol, int maxiter, int solver, double* corr,
                                dwf_solve_info* info)
{
    if (!c || c->kind != 1 || !thetas || !corr || nconf < 1 || src_t < 0 || src_t >= c->L.Nt ||
        src_x < 0 || src_x >= c->L.Nx)
        return DWF_BAD_ARG;
    CK(cudaSetDevice(c->device));
    int st = set_gauge(c, nconf, thetas, cudaMemcpyHostToDevice);
    if (st)
        return st;
    const long nrhs = 2L * nconf;
    const long fs = c->fsz();
    if ((st = ensure_workspace(c, int(nrhs))) ||
        (st = reserve(c, c->m_red, c->m_red_cap, size_t(nrhs) * c->L.Nt * 2)))
        return st;
    double2* const src = c->w_src;
    double2* const x = c->w_x;
    SrcDesc sd{};
    sd.L = c->L;
    sd.R = 2;
    sd.ls_src = 0;
    sd.src_x = src_x;
    sd.wil_t = src_t;
    sources_kernel<<<std::max(1, 8 * c->nsm), 256, 0, c->stream>>>(sd, nrhs, src);
    c->launches += 1;
    std::vector<int> conf(nrhs);
    for (long j = 0; j < nrhs; ++j)
        conf[j] = int(j / 2);
    std::vector<dwf_solve_info> inf(nrhs);
    st = propagators(c, int(nrhs), conf.data(), src, x, tol, maxiter, solver, inf.data());
    if (st)
        return st;
    for (long j = 0; j < nrhs; ++j)
        if (!std::isfinite(inf[j].true_relres) || inf[j].true_relres > 20.0 * tol)
        {
            char msg[200];
            std::snprintf(msg, sizeof msg,
                          "CGNR failed: iterations=%d, normal residual=%e, D residual=%e",
                          inf[j].iterations, inf[j].true_relres, inf[j].dirac_relres);
            return ctx_fail(c, DWF_NOT_CONVERGED, msg);
        }
    for (long j = 0; j < nrhs; j += 65535)
    {
        const int n = int(std::min<long>(65535, nrhs - j));
        contract_kernel<<<dim3(c->L.Nt, n), 128, 2 * c->L.Nx * sizeof(double), c->stream>>>(
            c->L, 0, 0, x + j * fs, c->m_red + j * c->L.Nt * 2);
        c->launches += 1;
    }
    std::vector<double> red(nrhs * c->L.Nt * 2);
    cudaMemcpyAsync(red.data(), c->m_red, red.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess)
        return ctx_fail(c, DWF_CUDA_ERROR, "correlator: copy-back failed");
    for (int cf = 0; cf < nconf; ++cf)
        for (int t = 0; t < c->L.Nt; ++t)
            corr[long(cf) * c->L.Nt + t] =
                red[((2L * cf) * c->L.Nt + t) * 2] + red[((2L * cf + 1) * c->L.Nt + t) * 2];
    if (info)
        std::copy(inf.begin(), inf.end(), info);
    return DWF_OK;
}

}  // extern "C"
