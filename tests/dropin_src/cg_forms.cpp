// Exercises the two forms of the drop-in conjugate_gradient on the GPU
// (three_part_dwf_study_b200/host/dropin/domain_wall/cg_solver.hpp): the named
// operator, the reference-shaped std::function form holding a
// b200::NormalOperator, and the std::function form holding the caller's own
// lambda (host recurrences around apply_D_dagger_D). Reads ./parameters.txt
// like the reference's mains; prints one line per form:
//   <form> <iterations> <converged> <relative residual> <|x - x_named| / |x_named|>
#include <cstdio>
#include <random>

#include "cg_solver.hpp"

int main()
{
    std::mt19937_64 rng(20240611ull);
    std::uniform_real_distribution<double> angle(-pi, pi);
    std::normal_distribution<double> normal(0.0, 1.0);
    Gauge theta(Ngauge);
    for (double& t : theta)
        t = angle(rng);
    VectorC b(Ndof);
    for (int i = 0; i < Ndof; ++i)
        b[i] = Complex(normal(rng), normal(rng));
    const double rtol = 1e-12;
    const CgResult named = conjugate_gradient(DWF_OP_DDAGD, theta, b, nullptr, rtol, 5000);
    const std::function<VectorC(const VectorC&)> tagged = b200::NormalOperator{DWF_OP_DDAGD, theta};
    const CgResult viaop = conjugate_gradient(tagged, b, nullptr, rtol, 5000);
    const CgResult lambda = conjugate_gradient(
        [&](const VectorC& v) { return apply_D_dagger_D(theta, v); }, b, nullptr, rtol, 5000);
    const double nx = named.x.norm();
    for (const auto& [name, r] : {std::pair<const char*, const CgResult*>{"named", &named},
                                  {"normal_operator", &viaop},
                                  {"lambda", &lambda}})
        std::printf("%s %d %d %.17g %.17g\n", name, r->iterations, int(r->converged),
                    r->relative_residual, (r->x - named.x).norm() / nx);
    return 0;
}
