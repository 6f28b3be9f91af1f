"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/liboracle.so (built by ``make -C oracle oracle``). Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, to
check GPU results or as the timed CPU baseline; the product never does.

Complex arrays are numpy complex128 in the reference layouts:
DWF fields  : flat [Ls*Nt*Nx*2], index ((s*Nt+t)*Nx+x)*2+spin
Wilson field: flat [Nt*Nx*2],    index (t*Nx+x)*2+spin
gauge theta : flat [2*Nt*Nx],    index (mu*Nt+t)*Nx+x
"""
import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None

D, DDAG, DDDAG, DDAGD = 0, 1, 2, 3


class DwfParams(C.Structure):
    _fields_ = [("Nt", C.c_int), ("Nx", C.c_int), ("Ls", C.c_int),
                ("M5", C.c_double), ("mf", C.c_double)]


class WilParams(C.Structure):
    _fields_ = [("Nt", C.c_int), ("Nx", C.c_int), ("m0", C.c_double),
                ("bc_t", C.c_double), ("bc_x", C.c_double)]


def lib():
    global _LIB
    if _LIB is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            import subprocess
            subprocess.run(["make", "-C", str(_HERE), "oracle"], check=True,
                           env=dict(os.environ))
        _LIB = C.CDLL(str(path))
    return _LIB


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c128(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


class Dwf:
    def __init__(self, Nt, Nx, Ls, M5, mf):
        self.p = DwfParams(Nt, Nx, Ls, M5, mf)
        self.Nt, self.Nx, self.Ls = Nt, Nx, Ls
        self.ndof = Ls * Nt * Nx * 2
        self.ngauge = 2 * Nt * Nx

    def apply(self, op, theta, v):
        v = _c128(v)
        out = np.empty(self.ndof, np.complex128)
        th = np.ascontiguousarray(theta, np.float64).ravel()
        lib().orc_dwf_apply(C.byref(self.p), op, _d(th), _d(v), _d(out))
        return out

    def cg(self, op, theta, b, rtol, maxiter, guess=None):
        b = _c128(b)
        th = np.ascontiguousarray(theta, np.float64).ravel()
        x = np.empty(self.ndof, np.complex128)
        it = C.c_int()
        rr = C.c_double()
        g = _c128(guess) if guess is not None else None
        st = lib().orc_dwf_cg(C.byref(self.p), op, _d(th), _d(b),
                              _d(g) if g is not None else None,
                              C.c_double(rtol), maxiter, _d(x), C.byref(it), C.byref(rr))
        return x, it.value, rr.value, st

    def pf_action_force(self, theta, phi, rtol, maxiter, guess=None):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        phi = _c128(phi)
        g = _c128(guess) if guess is not None else None
        act = C.c_double()
        force = np.empty(self.ngauge)
        eta = np.empty(self.ndof, np.complex128)
        it = C.c_int()
        rr = C.c_double()
        st = lib().orc_dwf_pf_action_force(C.byref(self.p), _d(th), _d(phi),
                                           _d(g) if g is not None else None,
                                           C.c_double(rtol), maxiter, C.byref(act),
                                           _d(force), _d(eta), C.byref(it), C.byref(rr))
        return dict(status=st, action=act.value, force=force, eta=eta,
                    iterations=it.value, relres=rr.value)

    def trajectory(self, beta, eps, nsteps, rtol, maxiter, theta0, chi, mom):
        th = np.ascontiguousarray(theta0, np.float64).ravel()
        chi = _c128(chi)
        mom = np.ascontiguousarray(mom, np.float64).ravel()
        out = np.empty(self.ngauge)
        info = np.empty(6)
        st = lib().orc_dwf_trajectory(C.byref(self.p), C.c_double(beta), C.c_double(eps),
                                      nsteps, C.c_double(rtol), maxiter, _d(th), _d(chi),
                                      _d(mom), _d(out), _d(info))
        return st, out, dict(dH=info[0], H0=info[1], H=info[2], Sg=info[3], Spf=info[4],
                             iterations=int(info[5]))

    def wall_propagator(self, theta, t_src, rtol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        psi = np.empty(2 * self.ndof, np.complex128)
        info = np.empty(8)
        st = lib().orc_dwf_wall_propagator(C.byref(self.p), _d(th), t_src, C.c_double(rtol),
                                           maxiter, _d(psi), _d(info))
        return st, psi.reshape(2, self.ndof), info.reshape(2, 4)

    def cpp_cj5(self, theta, rtol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        cpp = np.empty(self.Nt)
        cj5 = np.empty(self.Nt)
        st = lib().orc_dwf_cpp_cj5(C.byref(self.p), _d(th), C.c_double(rtol), maxiter,
                                   _d(cpp), _d(cj5))
        return st, cpp, cj5

    def momentum_cpp(self, theta, max_momentum, rtol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        out = np.empty((max_momentum + 1) * self.Nt)
        st = lib().orc_dwf_momentum_cpp(C.byref(self.p), _d(th), max_momentum,
                                        C.c_double(rtol), maxiter, _d(out))
        return st, out.reshape(max_momentum + 1, self.Nt)

    def loop(self, theta, seed, nnoise, rtol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        out = np.empty(self.Nt * self.Nx, np.complex128)
        st = lib().orc_dwf_loop(C.byref(self.p), _d(th), C.c_ulonglong(seed), nnoise,
                                C.c_double(rtol), maxiter, _d(out))
        return st, out


def gauge_action_force(Nt, Nx, beta, theta):
    th = np.ascontiguousarray(theta, np.float64).ravel()
    act = C.c_double()
    force = np.empty(2 * Nt * Nx)
    lib().orc_gauge_action_force(Nt, Nx, C.c_double(beta), _d(th), C.byref(act), _d(force))
    return act.value, force


def average_plaquette(Nt, Nx, theta):
    th = np.ascontiguousarray(theta, np.float64).ravel()
    f = lib().orc_average_plaquette
    f.restype = C.c_double
    return f(Nt, Nx, _d(th))


def rng_z4(seed, n):
    out = np.empty(n, np.int32)
    lib().orc_rng_z4(C.c_ulonglong(seed), C.c_long(n), out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def rng_normals(seed, n):
    out = np.empty(n)
    lib().orc_rng_normals(C.c_ulonglong(seed), C.c_long(n), _d(out))
    return out


def dwf_draws(seed, ntraj, ndof, ngauge):
    chi = np.empty((ntraj, ndof), np.complex128)
    mom = np.empty((ntraj, ngauge))
    u = np.empty(ntraj)
    lib().orc_dwf_draws(C.c_ulonglong(seed), ntraj, ndof, ngauge, _d(chi), _d(mom), _d(u))
    return chi, mom, u


def wil_draws(seed, ntraj, ntot, ngauge):
    mom = np.empty((ntraj, ngauge))
    chi = np.empty((ntraj, ntot), np.complex128)
    u = np.empty(ntraj)
    lib().orc_wil_draws(C.c_ulonglong(seed), ntraj, ntot, ngauge, _d(mom), _d(chi), _d(u))
    return mom, chi, u


class Wilson:
    def __init__(self, Nt, Nx, m0, bc_t=-1.0, bc_x=1.0):
        self.p = WilParams(Nt, Nx, m0, bc_t, bc_x)
        self.Nt, self.Nx = Nt, Nx
        self.ntot = Nt * Nx * 2
        self.ngauge = 2 * Nt * Nx

    def apply(self, op, theta, v):
        v = _c128(v)
        th = np.ascontiguousarray(theta, np.float64).ravel()
        out = np.empty(self.ntot, np.complex128)
        lib().orc_wil_apply(C.byref(self.p), op, _d(th), _d(v), _d(out))
        return out

    def cg(self, op, theta, b, tol, maxiter):
        b = _c128(b)
        th = np.ascontiguousarray(theta, np.float64).ravel()
        x = np.empty(self.ntot, np.complex128)
        it = C.c_int()
        rr = C.c_double()
        st = lib().orc_wil_cg(C.byref(self.p), op, _d(th), _d(b), C.c_double(tol), maxiter,
                              _d(x), C.byref(it), C.byref(rr))
        return x, it.value, rr.value, st

    def solve_cgnr(self, theta, source, tol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        src = _c128(source)
        x = np.empty(self.ntot, np.complex128)
        info = np.empty(3)
        st = lib().orc_wil_solve_cgnr(C.byref(self.p), _d(th), _d(src), C.c_double(tol),
                                      maxiter, _d(x), _d(info))
        return st, x, info

    def solve_dddag(self, theta, phi, tol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        phi = _c128(phi)
        eta = np.empty(self.ntot, np.complex128)
        res = C.c_double()
        st = lib().orc_wil_solve_dddag(C.byref(self.p), _d(th), _d(phi), C.c_double(tol),
                                       maxiter, _d(eta), C.byref(res))
        return st, eta, res.value

    def pf_action_force(self, theta, phi, tol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        phi = _c128(phi)
        act = C.c_double()
        force = np.empty(self.ngauge)
        st = lib().orc_wil_pf_action_force(C.byref(self.p), _d(th), _d(phi), C.c_double(tol),
                                           maxiter, C.byref(act), _d(force))
        return st, act.value, force

    def hmc_step(self, beta, eps, nsteps, tol, maxiter, theta_old, mom, chi, u):
        th = np.ascontiguousarray(theta_old, np.float64).ravel()
        mom = np.ascontiguousarray(mom, np.float64).ravel()
        chi = _c128(chi)
        out = np.empty(self.ngauge)
        info = np.empty(3)
        st = lib().orc_wil_hmc_step(C.byref(self.p), C.c_double(beta), C.c_double(eps), nsteps,
                                    C.c_double(tol), maxiter, _d(th), _d(mom), _d(chi),
                                    C.c_double(u), _d(out), _d(info))
        return st, out, dict(dH=info[0], pacc=info[1], accepted=bool(info[2]))

    def correlator(self, theta, src_t, src_x, tol, maxiter):
        th = np.ascontiguousarray(theta, np.float64).ravel()
        out = np.empty(self.Nt)
        st = lib().orc_wil_correlator(C.byref(self.p), _d(th), src_t, src_x, C.c_double(tol),
                                      maxiter, _d(out))
        return st, out
