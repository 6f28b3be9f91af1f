// Drop-in for domain_wall/include/gauge.hpp (gauge action, force and
// plaquette on the GPU, FP64).
#pragma once

#include "b200_dwf.hpp"
#include "indexing.hpp"

struct GaugeActionForce
{
    double action;
    Gauge force;
};

inline double plaquette_angle(const Gauge& theta, int t, int x)
{
    const int tp = plus_periodic(t, Nt);
    const int xp = plus_periodic(x, Nx);
    return theta[gauge_index(0, t, x)] + theta[gauge_index(1, tp, x)] -
           theta[gauge_index(0, t, xp)] - theta[gauge_index(1, t, x)];
}

inline GaugeActionForce gauge_action_force(const Gauge& theta)
{
    dwf_ctx* c = b200_dwf_context();
    GaugeActionForce r{0.0, Gauge(Ngauge, 0.0)};
    b200::check(c, dwf_gauge_action_force(c, theta.data(), &r.action, r.force.data()));
    return r;
}

inline double average_plaquette(const Gauge& theta)
{
    dwf_ctx* c = b200_dwf_context();
    double p = 0.0;
    b200::check(c, dwf_average_plaquette(c, theta.data(), &p));
    return p;
}
