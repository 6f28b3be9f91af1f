// CPU oracle (TEST INFRASTRUCTURE ONLY): a restatement of the reference's
// Wilson and domain-wall arithmetic with explicit parameters. See oracle.h for
// the layouts. Each function names the reference lines it follows; operations
// are written in the reference's order so that, compiled without FMA
// contraction, results match the reference build bit for bit where the
// reference's own vector helpers sum sequentially.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <random>
#include <vector>

namespace {

using C = std::complex<double>;
using Field = std::vector<C>;

struct Dwf
{
    int Nt, Nx, Ls;
    double M5, mf;
    int V() const { return Nt * Nx; }
    int ndof() const { return Ls * Nt * Nx * 2; }
    // domain_wall/include/indexing.hpp:5-13
    int fi(int s, int t, int x, int a) const { return ((s * Nt + t) * Nx + x) * 2 + a; }
    int gi(int mu, int t, int x) const { return (mu * Nt + t) * Nx + x; }
};

inline int pp(int x, int n) { return (x + 1) % n; }      // indexing.hpp:15-18
inline int mp(int x, int n) { return (x - 1 + n) % n; }  // indexing.hpp:20-23

Field to_field(const double* d, long n)
{
    Field f(n);
    for (long i = 0; i < n; ++i)
        f[i] = C(d[2 * i], d[2 * i + 1]);
    return f;
}

void from_field(const Field& f, double* d)
{
    for (std::size_t i = 0; i < f.size(); ++i)
    {
        d[2 * i] = f[i].real();
        d[2 * i + 1] = f[i].imag();
    }
}

C link(const double* theta, int idx) { return std::exp(C(0.0, theta[idx])); }  // dwf_operator.hpp:10-13

C cdot(const Field& a, const Field& b)  // a^dag b, summed in index order
{
    C s(0.0, 0.0);
    for (std::size_t i = 0; i < a.size(); ++i)
        s += std::conj(a[i]) * b[i];
    return s;
}

double sqnorm(const Field& a)
{
    double s = 0.0;
    for (const C& v : a)
        s += std::norm(v);
    return s;
}

// (I - s1) v, (I + s1) v, (I - s2) v, (I + s2) v with s1 = [[0,1],[1,0]],
// s2 = [[0,-i],[i,0]] (domain_wall/include/spin.hpp:5-19). Products with the
// entries 0, +-1, +-i are exact, so these match a 2x2 matrix-vector product.
inline void i_minus_s1(const C* v, C* o) { o[0] = v[0] - v[1]; o[1] = -v[0] + v[1]; }
inline void i_plus_s1(const C* v, C* o) { o[0] = v[0] + v[1]; o[1] = v[0] + v[1]; }
inline void i_minus_s2(const C* v, C* o)
{
    o[0] = v[0] + C(0, 1) * v[1];
    o[1] = C(0, -1) * v[0] + v[1];
}
inline void i_plus_s2(const C* v, C* o)
{
    o[0] = v[0] + C(0, -1) * v[1];
    o[1] = C(0, 1) * v[0] + v[1];
}

// apply_D (dwf_operator.hpp:15-92) and apply_D_dagger (:94-171).
Field dwf_D(const Dwf& g, const double* theta, const Field& psi, bool dag)
{
    Field out(psi.size());
    for (std::size_t i = 0; i < psi.size(); ++i)
        out[i] = (3.0 - g.M5) * psi[i];
    for (int s = 0; s < g.Ls; ++s)
        for (int t = 0; t < g.Nt; ++t)
        {
            const int tp = pp(t, g.Nt), tm = mp(t, g.Nt);
            const double sign_tp = (t == g.Nt - 1) ? -1.0 : 1.0;
            const double sign_tm = (t == 0) ? -1.0 : 1.0;
            for (int x = 0; x < g.Nx; ++x)
            {
                const int xp = pp(x, g.Nx), xm = mp(x, g.Nx);
                C v_tp[2], v_tm[2], v_xp[2], v_xm[2];
                for (int a = 0; a < 2; ++a)
                {
                    v_tp[a] = sign_tp * psi[g.fi(s, tp, x, a)];
                    v_tm[a] = sign_tm * psi[g.fi(s, tm, x, a)];
                    v_xp[a] = psi[g.fi(s, t, xp, a)];
                    v_xm[a] = psi[g.fi(s, t, xm, a)];
                }
                const C Ut = link(theta, g.gi(0, t, x));
                const C Ut_dag = std::conj(link(theta, g.gi(0, tm, x)));
                const C Ux = link(theta, g.gi(1, t, x));
                const C Ux_dag = std::conj(link(theta, g.gi(1, t, xm)));
                C term_tp[2], term_tm[2], term_xp[2], term_xm[2];
                if (!dag)
                {
                    i_minus_s1(v_tp, term_tp);
                    i_plus_s1(v_tm, term_tm);
                    i_minus_s2(v_xp, term_xp);
                    i_plus_s2(v_xm, term_xm);
                    for (int a = 0; a < 2; ++a)
                    {
                        const int row = g.fi(s, t, x, a);
                        out[row] += -0.5 * Ut * term_tp[a];
                        out[row] += -0.5 * Ut_dag * term_tm[a];
                        out[row] += -0.5 * Ux * term_xp[a];
                        out[row] += -0.5 * Ux_dag * term_xm[a];
                    }
                    const int r1 = g.fi(s, t, x, 1);
                    if (s < g.Ls - 1)
                        out[r1] += -psi[g.fi(s + 1, t, x, 1)];
                    else
                        out[r1] += g.mf * psi[g.fi(0, t, x, 1)];
                    const int r0 = g.fi(s, t, x, 0);
                    if (s > 0)
                        out[r0] += -psi[g.fi(s - 1, t, x, 0)];
                    else
                        out[r0] += g.mf * psi[g.fi(g.Ls - 1, t, x, 0)];
                }
                else
                {
                    i_minus_s1(v_tm, term_tm);
                    i_plus_s1(v_tp, term_tp);
                    i_minus_s2(v_xm, term_xm);
                    i_plus_s2(v_xp, term_xp);
                    for (int a = 0; a < 2; ++a)
                    {
                        const int row = g.fi(s, t, x, a);
                        out[row] += -0.5 * Ut_dag * term_tm[a];
                        out[row] += -0.5 * Ut * term_tp[a];
                        out[row] += -0.5 * Ux_dag * term_xm[a];
                        out[row] += -0.5 * Ux * term_xp[a];
                    }
                    const int r1 = g.fi(s, t, x, 1);
                    if (s > 0)
                        out[r1] += -psi[g.fi(s - 1, t, x, 1)];
                    else
                        out[r1] += g.mf * psi[g.fi(g.Ls - 1, t, x, 1)];
                    const int r0 = g.fi(s, t, x, 0);
                    if (s < g.Ls - 1)
                        out[r0] += -psi[g.fi(s + 1, t, x, 0)];
                    else
                        out[r0] += g.mf * psi[g.fi(0, t, x, 0)];
                }
            }
        }
    return out;
}

Field dwf_op(const Dwf& g, int op, const double* theta, const Field& v)
{
    switch (op)
    {
    case ORC_D: return dwf_D(g, theta, v, false);
    case ORC_DDAG: return dwf_D(g, theta, v, true);
    case ORC_DDDAG: return dwf_D(g, theta, dwf_D(g, theta, v, true), false);  // dwf_operator.hpp:173-176
    default: return dwf_D(g, theta, dwf_D(g, theta, v, false), true);       // dwf_operator.hpp:178-181
    }
}

struct CgOut
{
    Field x;
    int iterations;
    double relres;
    int status;  // 0 converged, 1 not converged, 2 zero denominator
};

// conjugate_gradient (domain_wall/include/cg_solver.hpp:17-64).
template <typename A>
CgOut cg(const A& apply, const Field& b, const Field* guess, double rtol, int maxiter)
{
    Field x = guess ? *guess : Field(b.size(), C(0.0, 0.0));
    Field r = apply(x);
    for (std::size_t i = 0; i < r.size(); ++i)
        r[i] = b[i] - r[i];
    Field p = r;
    const double bnorm = std::sqrt(sqnorm(b));
    if (bnorm == 0.0)
        return {x, 0, 0.0, 0};
    double rr_old = std::real(cdot(r, r));
    double rel = std::sqrt(rr_old) / bnorm;
    if (rel <= rtol)
        return {x, 0, rel, 0};
    for (int it = 1; it <= maxiter; ++it)
    {
        const Field Ap = apply(p);
        const C den = cdot(p, Ap);
        if (std::abs(den) == 0.0)
            return {x, it, rel, 2};
        const double alpha = rr_old / std::real(den);
        for (std::size_t i = 0; i < x.size(); ++i)
            x[i] += alpha * p[i];
        for (std::size_t i = 0; i < x.size(); ++i)
            r[i] -= alpha * Ap[i];
        const double rr_new = std::real(cdot(r, r));
        rel = std::sqrt(rr_new) / bnorm;
        if (rel <= rtol)
            return {x, it, rel, 0};
        const double beta_cg = rr_new / rr_old;
        for (std::size_t i = 0; i < x.size(); ++i)
            p[i] = r[i] + beta_cg * p[i];
        rr_old = rr_new;
    }
    return {x, maxiter, rel, 1};
}

struct PfOut
{
    double action;
    std::vector<double> force;
    Field eta;
    int iterations;
    double relres;
    int status;
};

// pseudofermion_action_force (domain_wall/include/pseudofermion.hpp:22-166).
PfOut dwf_pf(const Dwf& g, const double* theta, const Field& phi, const Field* guess,
             double rtol, int maxiter)
{
    const auto M = [&](const Field& v) { return dwf_op(g, ORC_DDDAG, theta, v); };
    CgOut sol = cg(M, phi, guess, rtol, maxiter);
    PfOut o{0.0, std::vector<double>(2 * g.V(), 0.0), sol.x, sol.iterations, sol.relres,
            sol.status};
    if (sol.status != 0)
        return o;
    const Field& eta = sol.x;
    o.action = std::real(cdot(phi, eta));
    const Field xi = dwf_D(g, theta, eta, true);
    const int V = g.V();
    std::vector<C> t_fwd(V), t_bwd(V), x_fwd(V), x_bwd(V);
    for (int t = 0; t < g.Nt; ++t)
    {
        const int tp = pp(t, g.Nt), tm = mp(t, g.Nt);
        const double sign_tp = (t == g.Nt - 1) ? -1.0 : 1.0;
        const double sign_tm = (t == 0) ? -1.0 : 1.0;
        for (int x = 0; x < g.Nx; ++x)
        {
            const int xp = pp(x, g.Nx), xm = mp(x, g.Nx);
            C tf = 0.0, tb = 0.0, xf = 0.0, xb = 0.0;
            for (int s = 0; s < g.Ls; ++s)
            {
                C xi_tp[2], xi_tm[2], xi_xp[2], xi_xm[2], eh[2];
                for (int a = 0; a < 2; ++a)
                {
                    xi_tp[a] = sign_tp * xi[g.fi(s, tp, x, a)];
                    xi_tm[a] = sign_tm * xi[g.fi(s, tm, x, a)];
                    xi_xp[a] = xi[g.fi(s, t, xp, a)];
                    xi_xm[a] = xi[g.fi(s, t, xm, a)];
                    eh[a] = eta[g.fi(s, t, x, a)];
                }
                C ttf[2], ttb[2], txf[2], txb[2];
                i_minus_s1(xi_tp, ttf);
                i_plus_s1(xi_tm, ttb);
                i_minus_s2(xi_xp, txf);
                i_plus_s2(xi_xm, txb);
                const C Ut = std::exp(C(0.0, theta[g.gi(0, t, x)]));
                const C Ut_dag = std::conj(std::exp(C(0.0, theta[g.gi(0, tm, x)])));
                const C Ux = std::exp(C(0.0, theta[g.gi(1, t, x)]));
                const C Ux_dag = std::conj(std::exp(C(0.0, theta[g.gi(1, t, xm)])));
                for (int a = 0; a < 2; ++a)
                {
                    const C es = std::conj(eh[a]);
                    tf += es * (C(0.0, -0.5) * Ut * ttf[a]);
                    tb += es * (C(0.0, 0.5) * Ut_dag * ttb[a]);
                    xf += es * (C(0.0, -0.5) * Ux * txf[a]);
                    xb += es * (C(0.0, 0.5) * Ux_dag * txb[a]);
                }
            }
            t_fwd[t * g.Nx + x] = tf;
            t_bwd[t * g.Nx + x] = tb;
            x_fwd[t * g.Nx + x] = xf;
            x_bwd[t * g.Nx + x] = xb;
        }
    }
    for (int t = 0; t < g.Nt; ++t)
    {
        const int tp = pp(t, g.Nt);
        for (int x = 0; x < g.Nx; ++x)
        {
            const int xp = pp(x, g.Nx);
            o.force[g.gi(0, t, x)] = -2.0 * std::real(t_fwd[t * g.Nx + x] + t_bwd[tp * g.Nx + x]);
            o.force[g.gi(1, t, x)] = -2.0 * std::real(x_fwd[t * g.Nx + x] + x_bwd[t * g.Nx + xp]);
        }
    }
    return o;
}

// plaquette_angle (domain_wall/include/gauge.hpp:15-24; wilson/include/gauge.hpp:20-27).
double plaq_angle(int Nt, int Nx, const double* th, int t, int x)
{
    const int tp = pp(t, Nt), xp = pp(x, Nx);
    return th[(0 * Nt + t) * Nx + x] + th[(1 * Nt + tp) * Nx + x] - th[(0 * Nt + t) * Nx + xp] -
           th[(1 * Nt + t) * Nx + x];
}

// gauge_action_force (domain_wall/include/gauge.hpp:26-62; wilson/include/gauge.hpp:38-62).
double gauge_af(int Nt, int Nx, double beta, const double* th, double* force)
{
    double action = 0.0;
    std::vector<double> sp(Nt * Nx);
    for (int t = 0; t < Nt; ++t)
        for (int x = 0; x < Nx; ++x)
        {
            const double p = plaq_angle(Nt, Nx, th, t, x);
            action += beta * (1.0 - std::cos(p));
            sp[t * Nx + x] = std::sin(p);
        }
    for (int t = 0; t < Nt; ++t)
    {
        const int tm = mp(t, Nt);
        for (int x = 0; x < Nx; ++x)
        {
            const int xm = mp(x, Nx);
            const double here = sp[t * Nx + x];
            force[(0 * Nt + t) * Nx + x] = beta * (here - sp[t * Nx + xm]);
            force[(1 * Nt + t) * Nx + x] = beta * (sp[tm * Nx + x] - here);
        }
    }
    return action;
}

Dwf make(const orc_dwf_params* p) { return Dwf{p->Nt, p->Nx, p->Ls, p->M5, p->mf}; }

// projector_L = (1 - s3)/2 = diag(0, 1), projector_R = (1 + s3)/2 = diag(1, 0)
// (domain_wall/include/spin.hpp:33-42).
inline double PL(int a, int b) { return (a == b && a == 1) ? 1.0 : 0.0; }
inline double PR(int a, int b) { return (a == b && a == 0) ? 1.0 : 0.0; }

// ---- Wilson ----------------------------------------------------------------

struct Wil
{
    int Nt, Nx;
    double m0, bct, bcx;
    int ntot() const { return Nt * Nx * 2; }
    int si(int t, int x, int a) const { return (t * Nx + x) * 2 + a; }  // wilson/include/indexing.hpp:5-8
    int li(int mu, int t, int x) const { return (mu * Nt + t) * Nx + x; }
};

struct Sparse
{
    int n = 0;
    std::vector<std::vector<std::pair<int, C>>> rows;
    Field mul(const Field& v) const
    {
        Field out(n);
        for (int i = 0; i < n; ++i)
        {
            C s(0.0, 0.0);
            for (const auto& e : rows[i])
                s += e.second * v[e.first];
            out[i] = s;
        }
        return out;
    }
    Sparse adjoint() const
    {
        Sparse a;
        a.n = n;
        a.rows.assign(n, {});
        for (int i = 0; i < n; ++i)
            for (const auto& e : rows[i])
                a.rows[e.first].push_back({i, std::conj(e.second)});
        return a;
    }
    Sparse times(const Sparse& b) const
    {
        Sparse o;
        o.n = n;
        o.rows.assign(n, {});
        std::vector<C> acc(n);
        std::vector<char> used(n, 0);
        std::vector<int> cols;
        for (int i = 0; i < n; ++i)
        {
            cols.clear();
            for (const auto& ea : rows[i])
                for (const auto& eb : b.rows[ea.first])
                {
                    if (!used[eb.first])
                    {
                        used[eb.first] = 1;
                        acc[eb.first] = C(0.0, 0.0);
                        cols.push_back(eb.first);
                    }
                    acc[eb.first] += ea.second * eb.second;
                }
            std::sort(cols.begin(), cols.end());
            for (int c : cols)
            {
                o.rows[i].push_back({c, acc[c]});
                used[c] = 0;
            }
        }
        return o;
    }
};

// build_wilson_matrix (wilson/include/wilson_operator.hpp:10-62): diagonal
// (2+m0), hops -1/2 * bc * U * (I -+ gamma); entries with |value| = 0 skipped,
// duplicates summed in insertion order, rows sorted by column.
Sparse wilson_matrix(const Wil& w, const double* theta)
{
    Sparse D;
    D.n = w.ntot();
    D.rows.assign(D.n, {});
    const C gt[2][2] = {{0.0, 1.0}, {1.0, 0.0}};
    const C gx[2][2] = {{0.0, C(0, -1)}, {C(0, 1), 0.0}};
    auto add = [&](int rt, int rx, int ct, int cx, int kind, double sgn, C coeff) {
        // kind: 0 identity, 1 gamma_t, 2 gamma_x; matrix I + sgn*gamma (or I)
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
            {
                C m = (a == b) ? C(1.0, 0.0) : C(0.0, 0.0);
                if (kind == 1)
                    m = m + sgn * gt[a][b];
                if (kind == 2)
                    m = m + sgn * gx[a][b];
                const C value = coeff * m;
                if (std::abs(value) > 0.0)
                {
                    auto& r = D.rows[w.si(rt, rx, a)];
                    const int col = w.si(ct, cx, b);
                    bool merged = false;
                    for (auto& e : r)
                        if (e.first == col)
                        {
                            e.second += value;
                            merged = true;
                            break;
                        }
                    if (!merged)
                        r.push_back({col, value});
                }
            }
    };
    for (int t = 0; t < w.Nt; ++t)
        for (int x = 0; x < w.Nx; ++x)
        {
            add(t, x, t, x, 0, 0.0, C(2.0 + w.m0, 0.0));
            const int tp = (t + 1) % w.Nt;
            const double bctp = (t == w.Nt - 1) ? w.bct : 1.0;
            const C Ut = std::exp(C(0, theta[w.li(0, t, x)]));
            add(t, x, tp, x, 1, -1.0, -0.5 * bctp * Ut);
            const int tm = (t - 1 + w.Nt) % w.Nt;
            const double bctm = (t == 0) ? w.bct : 1.0;
            const C Utd = std::exp(C(0, -theta[w.li(0, tm, x)]));
            add(t, x, tm, x, 1, 1.0, -0.5 * bctm * Utd);
            const int xp = (x + 1) % w.Nx;
            const double bcxp = (x == w.Nx - 1) ? w.bcx : 1.0;
            const C Ux = std::exp(C(0, theta[w.li(1, t, x)]));
            add(t, x, t, xp, 2, -1.0, -0.5 * bcxp * Ux);
            const int xm = (x - 1 + w.Nx) % w.Nx;
            const double bcxm = (x == 0) ? w.bcx : 1.0;
            const C Uxd = std::exp(C(0, -theta[w.li(1, t, xm)]));
            add(t, x, t, xm, 2, 1.0, -0.5 * bcxm * Uxd);
        }
    for (auto& r : D.rows)
        std::stable_sort(r.begin(), r.end(),
                         [](const std::pair<int, C>& a, const std::pair<int, C>& b) {
                             return a.first < b.first;
                         });
    return D;
}

// Jacobi-preconditioned CG on an assembled matrix, x0 = 0, stop at
// |r|^2 < tol^2 |b|^2 (the solver behind wilson/include/cg_solver.hpp:24-31,58-64).
CgOut jacobi_cg(const Sparse& A, const Field& b, double tol, int maxiter)
{
    const int n = A.n;
    std::vector<C> invd(n, C(1.0, 0.0));
    for (int j = 0; j < n; ++j)
        for (const auto& e : A.rows[j])
            if (e.first == j && e.second != C(0.0, 0.0))
                invd[j] = C(1.0, 0.0) / e.second;
    Field x(n, C(0.0, 0.0)), r = b, p(n), z(n);
    const double bb = sqnorm(b);
    if (bb == 0.0)
        return {x, 0, 0.0, 0};
    const double thr = std::max(tol * tol * bb, 2.2250738585072014e-308);
    double rr = sqnorm(r);
    if (rr < thr)
        return {x, 0, std::sqrt(rr / bb), 0};
    for (int i = 0; i < n; ++i)
        p[i] = invd[i] * r[i];
    double rz = std::real(cdot(r, p));
    int it = 0;
    while (it < maxiter)
    {
        const Field q = A.mul(p);
        const C alpha = rz / cdot(p, q);
        for (int i = 0; i < n; ++i)
        {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        rr = sqnorm(r);
        if (rr < thr)
            break;
        for (int i = 0; i < n; ++i)
            z[i] = invd[i] * r[i];
        const double rz_old = rz;
        rz = std::real(cdot(r, z));
        const double beta = rz / rz_old;
        for (int i = 0; i < n; ++i)
            p[i] = z[i] + beta * p[i];
        ++it;
    }
    return {x, it, std::sqrt(rr / bb), rr < thr ? 0 : 1};
}

double rel_norm(const Field& a, const Field& b)  // |a - b| / max(|b|, 1e-300)
{
    double s = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i)
        s += std::norm(a[i] - b[i]);
    return std::sqrt(s) / std::max(std::sqrt(sqnorm(b)), 1.0e-300);
}

Wil makew(const orc_wil_params* p) { return Wil{p->Nt, p->Nx, p->m0, p->bc_t, p->bc_x}; }

// solve_DDdag (wilson/include/cg_solver.hpp:53-78) with its 20*tol guard.
int wil_dddag(const Wil& w, const double* theta, const Field& phi, double tol, int maxiter,
              Field& eta, double& residual)
{
    const Sparse D = wilson_matrix(w, theta);
    const Sparse A = D.times(D.adjoint());
    CgOut s = jacobi_cg(A, phi, tol, maxiter);
    eta = s.x;
    residual = rel_norm(A.mul(eta), phi);
    return (!std::isfinite(residual) || residual > 20.0 * tol) ? 1 : 0;
}

// pseudofermion_action_force (wilson/include/gauge.hpp:68-122).
int wil_pf(const Wil& w, const double* theta, const Field& phi, double tol, int maxiter,
           double& action, double* force)
{
    Field eta;
    double res = 0.0;
    const int st = wil_dddag(w, theta, phi, tol, maxiter, eta, res);
    if (st != 0)
        return st;
    const Sparse D = wilson_matrix(w, theta);
    const Field xi = D.adjoint().mul(eta);
    action = std::real(cdot(phi, eta));
    const int V2 = 2 * w.Nt * w.Nx;
    for (int i = 0; i < V2; ++i)
        force[i] = 0.0;
    for (int t = 0; t < w.Nt; ++t)
        for (int x = 0; x < w.Nx; ++x)
        {
            const int tp = (t + 1) % w.Nt, tm = (t - 1 + w.Nt) % w.Nt;
            const int xp = (x + 1) % w.Nx, xm = (x - 1 + w.Nx) % w.Nx;
            const double bctp = (t == w.Nt - 1) ? w.bct : 1.0;
            const double bctm = (t == 0) ? w.bct : 1.0;
            const double bcxp = (x == w.Nx - 1) ? w.bcx : 1.0;
            const double bcxm = (x == 0) ? w.bcx : 1.0;
            const C Ut = std::exp(C(0, theta[w.li(0, t, x)]));
            const C Utd = std::exp(C(0, -theta[w.li(0, tm, x)]));
            const C Ux = std::exp(C(0, theta[w.li(1, t, x)]));
            const C Uxd = std::exp(C(0, -theta[w.li(1, t, xm)]));
            C eh[2], xtp[2], xtm[2], xxp[2], xxm[2];
            for (int a = 0; a < 2; ++a)
            {
                eh[a] = eta[w.si(t, x, a)];
                xtp[a] = bctp * xi[w.si(tp, x, a)];
                xtm[a] = bctm * xi[w.si(tm, x, a)];
                xxp[a] = bcxp * xi[w.si(t, xp, a)];
                xxm[a] = bcxm * xi[w.si(t, xm, a)];
            }
            // (c * (I -+ gamma)) * v evaluated as a matrix product: each entry
            // c*m_ab, then sum over b in order.
            auto matvec = [](C c, int kind, double sgn, const C* v, C* o) {
                const C gt[2][2] = {{0.0, 1.0}, {1.0, 0.0}};
                const C gx[2][2] = {{0.0, C(0, -1)}, {C(0, 1), 0.0}};
                for (int a = 0; a < 2; ++a)
                {
                    C s(0.0, 0.0);
                    for (int b = 0; b < 2; ++b)
                    {
                        C m = ((a == b) ? C(1.0, 0.0) : C(0.0, 0.0)) +
                              sgn * (kind == 1 ? gt[a][b] : gx[a][b]);
                        s += (c * m) * v[b];
                    }
                    o[a] = s;
                }
            };
            C vt[2], vtb[2], vx[2], vxb[2];
            matvec(-0.5 * C(0, 1) * Ut, 1, -1.0, xtp, vt);
            matvec(0.5 * C(0, 1) * Utd, 1, 1.0, xtm, vtb);
            matvec(-0.5 * C(0, 1) * Ux, 2, -1.0, xxp, vx);
            matvec(0.5 * C(0, 1) * Uxd, 2, 1.0, xxm, vxb);
            auto dot2 = [](const C* a, const C* b) {
                return std::conj(a[0]) * b[0] + std::conj(a[1]) * b[1];
            };
            force[w.li(0, t, x)] += -2.0 * std::real(dot2(eh, vt));
            force[w.li(0, tm, x)] += -2.0 * std::real(dot2(eh, vtb));
            force[w.li(1, t, x)] += -2.0 * std::real(dot2(eh, vx));
            force[w.li(1, t, xm)] += -2.0 * std::real(dot2(eh, vxb));
        }
    return 0;
}

// wrap_angle (wilson/include/indexing.hpp:13-18)
double wrap_angle(double a)
{
    const double pi = 3.14159265358979323846;
    a = std::fmod(a + pi, 2.0 * pi);
    if (a < 0.0)
        a += 2.0 * pi;
    return a - pi;
}

}  // namespace

extern "C" {

void orc_dwf_apply(const orc_dwf_params* p, int op, const double* theta, const double* in,
                   double* out)
{
    const Dwf g = make(p);
    from_field(dwf_op(g, op, theta, to_field(in, g.ndof())), out);
}

int orc_dwf_cg(const orc_dwf_params* p, int op, const double* theta, const double* b,
               const double* guess, double rtol, int maxiter, double* x, int* iters,
               double* relres)
{
    const Dwf g = make(p);
    const Field bf = to_field(b, g.ndof());
    Field gf;
    if (guess)
        gf = to_field(guess, g.ndof());
    const auto A = [&](const Field& v) { return dwf_op(g, op, theta, v); };
    CgOut o = cg(A, bf, guess ? &gf : nullptr, rtol, maxiter);
    from_field(o.x, x);
    *iters = o.iterations;
    *relres = o.relres;
    return o.status;
}

int orc_dwf_pf_action_force(const orc_dwf_params* p, const double* theta, const double* phi,
                            const double* guess, double rtol, int maxiter, double* action,
                            double* force, double* eta, int* iters, double* relres)
{
    const Dwf g = make(p);
    Field gf;
    if (guess)
        gf = to_field(guess, g.ndof());
    PfOut o = dwf_pf(g, theta, to_field(phi, g.ndof()), guess ? &gf : nullptr, rtol, maxiter);
    *action = o.action;
    std::copy(o.force.begin(), o.force.end(), force);
    from_field(o.eta, eta);
    *iters = o.iterations;
    *relres = o.relres;
    return o.status;
}

void orc_gauge_action_force(int Nt, int Nx, double beta, const double* theta, double* action,
                            double* force)
{
    *action = gauge_af(Nt, Nx, beta, theta, force);
}

double orc_average_plaquette(int Nt, int Nx, const double* theta)
{
    // average_plaquette (domain_wall/include/gauge.hpp:64-73)
    double sum = 0.0;
    for (int t = 0; t < Nt; ++t)
        for (int x = 0; x < Nx; ++x)
            sum += std::cos(plaq_angle(Nt, Nx, theta, t, x));
    return sum / static_cast<double>(Nt * Nx);
}

// One domain-wall trajectory, restating domain_wall/generate_configs.cpp:56-160
// with chi and the momenta supplied by the caller.
int orc_dwf_trajectory(const orc_dwf_params* p, double beta, double eps, int nsteps, double rtol,
                       int maxiter, const double* theta0, const double* chi, const double* mom,
                       double* theta_out, double* out6)
{
    const Dwf g = make(p);
    const int NG = 2 * g.V();
    const Field phi = dwf_D(g, theta0, to_field(chi, g.ndof()), false);
    std::vector<double> momentum(mom, mom + NG);
    std::vector<double> fg(NG);
    const double sg0 = gauge_af(g.Nt, g.Nx, beta, theta0, fg.data());
    PfOut pf0 = dwf_pf(g, theta0, phi, nullptr, rtol, maxiter);
    if (pf0.status != 0)
        return pf0.status;
    long total_iters = pf0.iterations;
    Field eta_guess = pf0.eta;
    double k0 = 0.0;
    for (double v : momentum)
        k0 += 0.5 * v * v;
    const double H0 = k0 + sg0 + pf0.action;
    std::vector<double> theta(theta0, theta0 + NG), force(NG);
    for (int i = 0; i < NG; ++i)
        force[i] = fg[i] + pf0.force[i];
    for (int i = 0; i < NG; ++i)
        momentum[i] -= 0.5 * eps * force[i];
    double sg = sg0, spf = pf0.action;
    for (int step = 0; step < nsteps; ++step)
    {
        for (int i = 0; i < NG; ++i)
            theta[i] += eps * momentum[i];
        sg = gauge_af(g.Nt, g.Nx, beta, theta.data(), fg.data());
        PfOut pf = dwf_pf(g, theta.data(), phi, &eta_guess, rtol, maxiter);
        if (pf.status != 0)
            return pf.status;
        total_iters += pf.iterations;
        eta_guess = pf.eta;
        spf = pf.action;
        for (int i = 0; i < NG; ++i)
            force[i] = fg[i] + pf.force[i];
        if (step != nsteps - 1)
            for (int i = 0; i < NG; ++i)
                momentum[i] -= eps * force[i];
    }
    for (int i = 0; i < NG; ++i)
        momentum[i] -= 0.5 * eps * force[i];
    double k1 = 0.0;
    for (double v : momentum)
        k1 += 0.5 * v * v;
    const double H = k1 + sg + spf;
    std::copy(theta.begin(), theta.end(), theta_out);
    out6[0] = H - H0;
    out6[1] = H0;
    out6[2] = H;
    out6[3] = sg;
    out6[4] = spf;
    out6[5] = static_cast<double>(total_iters);
    return 0;
}

// boundary_wall_source_propagator (domain_wall/include/correlator.hpp:183-241).
int orc_dwf_wall_propagator(const orc_dwf_params* p, const double* theta, int t_src, double rtol,
                            int maxiter, double* psi_out, double* info8)
{
    const Dwf g = make(p);
    const auto M = [&](const Field& v) { return dwf_op(g, ORC_DDAGD, theta, v); };
    int status = 0;
    for (int b = 0; b < 2; ++b)
    {
        Field src(g.ndof(), C(0.0, 0.0));
        for (int x = 0; x < g.Nx; ++x)
            for (int a = 0; a < 2; ++a)
            {
                src[g.fi(0, t_src, x, a)] += PL(a, b);
                src[g.fi(g.Ls - 1, t_src, x, a)] += PR(a, b);
            }
        const Field rhs = dwf_D(g, theta, src, true);
        CgOut s = cg(M, rhs, nullptr, rtol, maxiter);
        if (s.status == 2)
            return 2;
        const Field Dx = dwf_D(g, theta, s.x, false);
        info8[4 * b + 0] = s.iterations;
        info8[4 * b + 1] = s.relres;
        info8[4 * b + 2] = rel_norm(Dx, src);
        info8[4 * b + 3] = s.status == 0 ? 1.0 : 0.0;
        from_field(s.x, psi_out + 2L * b * g.ndof());
        if (s.status != 0)
            status = 1;  // reported, not fatal (correlator.hpp:222-223)
    }
    return status;
}

// compute_CPP_CJ5 (domain_wall/include/correlator.hpp:243-310).
int orc_dwf_cpp_cj5(const orc_dwf_params* p, const double* theta, double rtol, int maxiter,
                    double* cpp, double* cj5)
{
    const Dwf g = make(p);
    for (int t = 0; t < g.Nt; ++t)
        cpp[t] = cj5[t] = 0.0;
    const int srcs[2] = {0, g.Nt / 2};
    std::vector<double> prop(4L * g.ndof());
    double info[8];
    for (int t_src : srcs)
    {
        const int st = orc_dwf_wall_propagator(p, theta, t_src, rtol, maxiter, prop.data(), info);
        if (st == 2)
            return 2;
        for (int t = 0; t < g.Nt; ++t)
        {
            const int dt = (t - t_src + g.Nt) % g.Nt;
            for (int x = 0; x < g.Nx; ++x)
                for (int b = 0; b < 2; ++b)
                {
                    const double* P = prop.data() + 2L * b * g.ndof();
                    C L[2], R[2], M[2], q[2];
                    for (int a = 0; a < 2; ++a)
                    {
                        L[a] = C(P[2 * g.fi(0, t, x, a)], P[2 * g.fi(0, t, x, a) + 1]);
                        R[a] = C(P[2 * g.fi(g.Ls - 1, t, x, a)],
                                 P[2 * g.fi(g.Ls - 1, t, x, a) + 1]);
                        M[a] = C(P[2 * g.fi(g.Ls / 2, t, x, a)],
                                 P[2 * g.fi(g.Ls / 2, t, x, a) + 1]);
                    }
                    // quark = PL*L + PR*R, as 2x2 products summed over the column index
                    for (int a = 0; a < 2; ++a)
                    {
                        C l(0.0, 0.0), r(0.0, 0.0);
                        for (int c = 0; c < 2; ++c)
                        {
                            l += PL(a, c) * L[c];
                            r += PR(a, c) * R[c];
                        }
                        q[a] = l + r;
                    }
                    cpp[dt] += std::norm(q[0]) + std::norm(q[1]);
                    for (int a = 0; a < 2; ++a)
                        cj5[dt] += std::real(std::conj(M[a]) * q[a]);
                }
        }
    }
    for (int t = 0; t < g.Nt; ++t)
    {
        cpp[t] /= 2.0;
        cj5[t] /= 2.0;
    }
    return 0;
}

// compute_momentum_CPP (domain_wall/include/correlator.hpp:111-181).
int orc_dwf_momentum_cpp(const orc_dwf_params* p, const double* theta, int max_momentum,
                         double rtol, int maxiter, double* out)
{
    const Dwf g = make(p);
    if (max_momentum < 0 || max_momentum > g.Nx / 2)
        return 6;
    for (int i = 0; i < (max_momentum + 1) * g.Nt; ++i)
        out[i] = 0.0;
    const auto M = [&](const Field& v) { return dwf_op(g, ORC_DDAGD, theta, v); };
    const int srcs[2] = {0, g.Nt / 2};
    const double pi = 3.141592653589793238462643383279502884;
    for (int t_src : srcs)
    {
        Field props[2];
        for (int b = 0; b < 2; ++b)
        {
            Field src(g.ndof(), C(0.0, 0.0));
            for (int a = 0; a < 2; ++a)
            {
                src[g.fi(0, t_src, 0, a)] += PL(a, b);
                src[g.fi(g.Ls - 1, t_src, 0, a)] += PR(a, b);
            }
            const Field rhs = dwf_D(g, theta, src, true);
            CgOut s = cg(M, rhs, nullptr, rtol, maxiter);
            if (s.status != 0)
                return s.status;
            props[b] = s.x;
        }
        for (int t = 0; t < g.Nt; ++t)
        {
            const int dt = (t - t_src + g.Nt) % g.Nt;
            for (int x = 0; x < g.Nx; ++x)
            {
                double local = 0.0;
                for (int b = 0; b < 2; ++b)
                {
                    C q[2];
                    for (int a = 0; a < 2; ++a)
                    {
                        C l(0.0, 0.0), r(0.0, 0.0);
                        for (int c = 0; c < 2; ++c)
                        {
                            l += PL(a, c) * props[b][g.fi(0, t, x, c)];
                            r += PR(a, c) * props[b][g.fi(g.Ls - 1, t, x, c)];
                        }
                        q[a] = l + r;
                    }
                    local += std::norm(q[0]) + std::norm(q[1]);
                }
                for (int n = 0; n <= max_momentum; ++n)
                {
                    const double pm = 2.0 * pi * n / g.Nx;
                    out[n * g.Nt + dt] += std::cos(pm * x) * local;
                }
            }
        }
    }
    for (int i = 0; i < (max_momentum + 1) * g.Nt; ++i)
        out[i] /= 2.0;
    return 0;
}

// estimate_pseudoscalar_loop_density (domain_wall/include/correlator.hpp:27-109).
int orc_dwf_loop(const orc_dwf_params* p, const double* theta, unsigned long long seed,
                 int nnoise, double rtol, int maxiter, double* loop)
{
    const Dwf g = make(p);
    if (nnoise < 1)
        return 6;
    const int V = g.V();
    std::vector<C> lp(V, C(0.0, 0.0));
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> z4(0, 3);
    const C phases[4] = {C(1.0, 0.0), C(0.0, 1.0), C(-1.0, 0.0), C(0.0, -1.0)};
    const auto M = [&](const Field& v) { return dwf_op(g, ORC_DDAGD, theta, v); };
    for (int k = 0; k < nnoise; ++k)
    {
        std::vector<C> eta(2L * V);
        Field src(g.ndof(), C(0.0, 0.0));
        for (int t = 0; t < g.Nt; ++t)
            for (int x = 0; x < g.Nx; ++x)
                for (int a = 0; a < 2; ++a)
                    eta[(t * g.Nx + x) * 2 + a] = phases[z4(rng)];
        for (int t = 0; t < g.Nt; ++t)
            for (int x = 0; x < g.Nx; ++x)
                for (int a = 0; a < 2; ++a)
                {
                    C l(0.0, 0.0), r(0.0, 0.0);
                    for (int c = 0; c < 2; ++c)
                    {
                        l += PL(a, c) * eta[(t * g.Nx + x) * 2 + c];
                        r += PR(a, c) * eta[(t * g.Nx + x) * 2 + c];
                    }
                    src[g.fi(0, t, x, a)] = l;
                    src[g.fi(g.Ls - 1, t, x, a)] += r;
                }
        const Field rhs = dwf_D(g, theta, src, true);
        CgOut s = cg(M, rhs, nullptr, rtol, maxiter);
        if (s.status != 0)
            return s.status;
        for (int t = 0; t < g.Nt; ++t)
            for (int x = 0; x < g.Nx; ++x)
            {
                C q[2];
                for (int a = 0; a < 2; ++a)
                {
                    C l(0.0, 0.0), r(0.0, 0.0);
                    for (int c = 0; c < 2; ++c)
                    {
                        l += PL(a, c) * s.x[g.fi(0, t, x, c)];
                        r += PR(a, c) * s.x[g.fi(g.Ls - 1, t, x, c)];
                    }
                    q[a] = l + r;
                }
                // noise.dot(gamma5 * q) with gamma5 = diag(1, -1)
                const C g5q0 = C(1.0, 0.0) * q[0] + C(0.0, 0.0) * q[1];
                const C g5q1 = C(0.0, 0.0) * q[0] + C(-1.0, 0.0) * q[1];
                lp[t * g.Nx + x] += std::conj(eta[(t * g.Nx + x) * 2]) * g5q0 +
                                    std::conj(eta[(t * g.Nx + x) * 2 + 1]) * g5q1;
            }
    }
    for (int i = 0; i < V; ++i)
    {
        lp[i] /= static_cast<double>(nnoise);
        loop[2 * i] = lp[i].real();
        loop[2 * i + 1] = lp[i].imag();
    }
    return 0;
}

void orc_rng_z4(unsigned long long seed, long n, int* digits)
{
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> z4(0, 3);
    for (long i = 0; i < n; ++i)
        digits[i] = z4(rng);
}

void orc_rng_normals(unsigned long long seed, long n, double* out)
{
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    for (long i = 0; i < n; ++i)
        out[i] = normal(rng);
}

// domain_wall/generate_configs.cpp:23-25, 56-69, 163: per trajectory chi[Ndof]
// as Complex(normal, normal)/sqrt(2) (the compiler draws the imaginary argument
// first), then the momenta, then one uniform for the Metropolis test.
void orc_dwf_draws(unsigned long long seed, int ntraj, int ndof, int ngauge, double* chi,
                   double* mom, double* u)
{
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    std::uniform_real_distribution<double> uniform(0.0, 1.0);
    for (int k = 0; k < ntraj; ++k)
    {
        for (int i = 0; i < ndof; ++i)
        {
            const double im = normal(rng);
            const double re = normal(rng);
            const C c = C(re, im) / std::sqrt(2.0);
            chi[2L * (long(k) * ndof + i)] = c.real();
            chi[2L * (long(k) * ndof + i) + 1] = c.imag();
        }
        for (int i = 0; i < ngauge; ++i)
            mom[long(k) * ngauge + i] = normal(rng);
        u[k] = uniform(rng);
    }
}

// wilson/include/gauge.hpp:16-18, 134-141, 178: momenta, then chi, then u.
void orc_wil_draws(unsigned long long seed, int ntraj, int ntot, int ngauge, double* mom,
                   double* chi, double* u)
{
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    std::uniform_real_distribution<double> uniform(0.0, 1.0);
    for (int k = 0; k < ntraj; ++k)
    {
        for (int i = 0; i < ngauge; ++i)
            mom[long(k) * ngauge + i] = normal(rng);
        for (int i = 0; i < ntot; ++i)
        {
            const double im = normal(rng);
            const double re = normal(rng);
            const C c = C(re, im) / std::sqrt(2.0);
            chi[2L * (long(k) * ntot + i)] = c.real();
            chi[2L * (long(k) * ntot + i) + 1] = c.imag();
        }
        u[k] = uniform(rng);
    }
}

void orc_wil_apply(const orc_wil_params* p, int op, const double* theta, const double* in,
                   double* out)
{
    const Wil w = makew(p);
    const Sparse D = wilson_matrix(w, theta);
    const Field v = to_field(in, w.ntot());
    Field r;
    switch (op)
    {
    case ORC_D: r = D.mul(v); break;
    case ORC_DDAG: r = D.adjoint().mul(v); break;
    case ORC_DDDAG: r = D.mul(D.adjoint().mul(v)); break;
    default: r = D.adjoint().mul(D.mul(v)); break;
    }
    from_field(r, out);
}

int orc_wil_cg(const orc_wil_params* p, int op, const double* theta, const double* b, double tol,
               int maxiter, double* x, int* iters, double* relres)
{
    const Wil w = makew(p);
    const Sparse D = wilson_matrix(w, theta);
    const Sparse A = (op == ORC_DDDAG) ? D.times(D.adjoint()) : D.adjoint().times(D);
    CgOut o = jacobi_cg(A, to_field(b, w.ntot()), tol, maxiter);
    from_field(o.x, x);
    *iters = o.iterations;
    *relres = o.relres;
    return o.status;
}

// solve_CGNR (wilson/include/cg_solver.hpp:19-51).
int orc_wil_solve_cgnr(const orc_wil_params* p, const double* theta, const double* source,
                       double tol, int maxiter, double* x, double* info3)
{
    const Wil w = makew(p);
    const Sparse D = wilson_matrix(w, theta);
    const Sparse Dd = D.adjoint();
    const Sparse N = Dd.times(D);
    const Field src = to_field(source, w.ntot());
    const Field rhs = Dd.mul(src);
    CgOut o = jacobi_cg(N, rhs, tol, maxiter);
    from_field(o.x, x);
    const double nres = rel_norm(N.mul(o.x), rhs);
    const double dres = rel_norm(D.mul(o.x), src);
    info3[0] = o.iterations;
    info3[1] = nres;
    info3[2] = dres;
    return (!std::isfinite(nres) || nres > 20.0 * tol) ? 1 : 0;
}

int orc_wil_solve_dddag(const orc_wil_params* p, const double* theta, const double* phi,
                        double tol, int maxiter, double* eta, double* residual)
{
    const Wil w = makew(p);
    Field e;
    const int st = wil_dddag(w, theta, to_field(phi, w.ntot()), tol, maxiter, e, *residual);
    from_field(e, eta);
    return st;
}

int orc_wil_pf_action_force(const orc_wil_params* p, const double* theta, const double* phi,
                            double tol, int maxiter, double* action, double* force)
{
    const Wil w = makew(p);
    return wil_pf(w, theta, to_field(phi, w.ntot()), tol, maxiter, *action, force);
}

// hmc_step (wilson/include/gauge.hpp:132-180) with the momenta, chi and the
// Metropolis uniform supplied by the caller.
int orc_wil_hmc_step(const orc_wil_params* p, double beta, double eps, int nsteps, double tol,
                     int maxiter, const double* theta_old, const double* mom, const double* chi,
                     double u, double* theta_out, double* info3)
{
    const Wil w = makew(p);
    const int NG = 2 * w.Nt * w.Nx;
    std::vector<double> momentum(mom, mom + NG);
    const Sparse D0 = wilson_matrix(w, theta_old);
    const Field phi = D0.mul(to_field(chi, w.ntot()));
    std::vector<double> Fg(NG), Fpf(NG), total(NG);
    const double old_Sg = gauge_af(w.Nt, w.Nx, beta, theta_old, Fg.data());
    double old_Spf = 0.0;
    int st = wil_pf(w, theta_old, phi, tol, maxiter, old_Spf, Fpf.data());
    if (st)
        return st;
    double old_K = 0.0;
    for (double v : momentum)
        old_K += v * v;
    old_K *= 0.5;
    std::vector<double> theta(theta_old, theta_old + NG);
    for (int i = 0; i < NG; ++i)
        total[i] = Fg[i] + Fpf[i];
    for (int i = 0; i < NG; ++i)
        momentum[i] -= 0.5 * eps * total[i];
    double dummy = 0.0;
    for (int step = 0; step < nsteps; ++step)
    {
        for (int i = 0; i < NG; ++i)
            theta[i] = wrap_angle(theta[i] + eps * momentum[i]);
        gauge_af(w.Nt, w.Nx, beta, theta.data(), Fg.data());
        st = wil_pf(w, theta.data(), phi, tol, maxiter, dummy, Fpf.data());
        if (st)
            return st;
        for (int i = 0; i < NG; ++i)
            total[i] = Fg[i] + Fpf[i];
        const double factor = (step == nsteps - 1) ? 0.5 : 1.0;
        for (int i = 0; i < NG; ++i)
            momentum[i] -= factor * eps * total[i];
    }
    const double new_Sg = gauge_af(w.Nt, w.Nx, beta, theta.data(), Fg.data());
    double new_Spf = 0.0;
    st = wil_pf(w, theta.data(), phi, tol, maxiter, new_Spf, Fpf.data());
    if (st)
        return st;
    double new_K = 0.0;
    for (double v : momentum)
        new_K += v * v;
    new_K *= 0.5;
    const double dH = (new_K + new_Sg + new_Spf) - (old_K + old_Sg + old_Spf);
    const double pacc = std::min(1.0, std::exp(-dH));
    const bool acc = u < pacc;
    for (int i = 0; i < NG; ++i)
        theta_out[i] = acc ? theta[i] : theta_old[i];
    info3[0] = dH;
    info3[1] = pacc;
    info3[2] = acc ? 1.0 : 0.0;
    return 0;
}

// pseudoscalar_correlator (wilson/include/correlator.hpp:10-40).
int orc_wil_correlator(const orc_wil_params* p, const double* theta, int src_t, int src_x,
                       double tol, int maxiter, double* corr)
{
    const Wil w = makew(p);
    std::vector<double> prop(2L * 2 * w.ntot());
    for (int b = 0; b < 2; ++b)
    {
        std::vector<double> src(2L * w.ntot(), 0.0);
        src[2 * w.si(src_t, src_x, b)] = 1.0;
        double info[3];
        const int st =
            orc_wil_solve_cgnr(p, theta, src.data(), tol, maxiter, prop.data() + 2L * b * w.ntot(),
                               info);
        if (st)
            return st;
    }
    for (int t = 0; t < w.Nt; ++t)
    {
        double c = 0.0;
        for (int x = 0; x < w.Nx; ++x)
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b)
                {
                    const double* P = prop.data() + 2L * b * w.ntot() + 2 * w.si(t, x, a);
                    c += P[0] * P[0] + P[1] * P[1];
                }
        corr[t] = c;
    }
    return 0;
}

}  // extern "C"
