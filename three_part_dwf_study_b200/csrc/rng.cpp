// Host random streams of the reference, reproduced with the same libstdc++
// engines and distributions so that heat-bath fields and Z4 noise are
// identical to the reference's draws.
#include <cmath>
#include <complex>
#include <cstdint>
#include <new>
#include <random>

#include "dwf_b200.h"

struct dwf_rng
{
    std::mt19937_64 engine;
    std::normal_distribution<double> normal{0.0, 1.0};
    std::uniform_real_distribution<double> uniform{0.0, 1.0};
    explicit dwf_rng(uint64_t seed) : engine(seed) {}
};

extern "C" {

int dwf_rng_create(uint64_t seed, dwf_rng** out)
{
    if (!out)
        return DWF_BAD_ARG;
    *out = new (std::nothrow) dwf_rng(seed);
    return *out ? DWF_OK : DWF_BAD_ARG;
}

int dwf_rng_destroy(dwf_rng* r)
{
    delete r;
    return DWF_OK;
}

int dwf_rng_normals(dwf_rng* r, long n, double* out)
{
    if (!r || n < 0 || (n > 0 && !out))
        return DWF_BAD_ARG;
    for (long i = 0; i < n; ++i)
        out[i] = r->normal(r->engine);
    return DWF_OK;
}

int dwf_rng_uniform(dwf_rng* r, double* out)
{
    if (!r || !out)
        return DWF_BAD_ARG;
    *out = r->uniform(r->engine);
    return DWF_OK;
}

int dwf_rng_pseudofermion(dwf_rng* r, long n, double* chi)
{
    if (!r || n < 0 || (n > 0 && !chi))
        return DWF_BAD_ARG;
    for (long i = 0; i < n; ++i)
    {
        // Complex(normal(rng), normal(rng)): the reference's compiler evaluates
        // the imaginary argument first.
        const double im = r->normal(r->engine);
        const double re = r->normal(r->engine);
        const std::complex<double> c = std::complex<double>(re, im) / std::sqrt(2.0);
        chi[2 * i] = c.real();
        chi[2 * i + 1] = c.imag();
    }
    return DWF_OK;
}

int dwf_z4_digits(uint64_t seed, long n, signed char* out)
{
    if (n < 0 || (n > 0 && !out))
        return DWF_BAD_ARG;
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> z4(0, 3);
    for (long i = 0; i < n; ++i)
        out[i] = static_cast<signed char>(z4(rng));
    return DWF_OK;
}

}  // extern "C"
