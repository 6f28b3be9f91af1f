"""Host-side mirror of the reference's Wilson entry points over the C ABI.

    build_wilson_matrix(theta) . v  -> apply_D / apply_D_dagger
        (wilson/include/wilson_operator.hpp:10-62, applied matrix-free)
    solve_CGNR, solve_DDdag          (wilson/include/cg_solver.hpp:19-78)
    gauge_action_force, pseudofermion_action_force, average_plaquette,
    hmc_step                         (wilson/include/gauge.hpp:20-180)
Fields: numpy complex128, index (t*Nx + x)*2 + spin; theta float64
(mu*Nt + t)*Nx + x. Errors raise RuntimeError with the reference's message.
"""
import ctypes as C

import numpy as np

from . import _capi as A
from .dwf import DomainWall, _ptr


class Wilson(DomainWall):
    """A Wilson context (wilson.Nt, wilson.Nx, wilson.m0, wilson.beta and the
    fermion boundary signs)."""

    def __init__(self, Nt, Nx, m0, beta=0.0, bc_t=-1.0, bc_x=1.0, device=0):
        self.Nt, self.Nx, self.Ls = int(Nt), int(Nx), 1
        self.m0, self.beta = float(m0), float(beta)
        self.bc_t, self.bc_x = float(bc_t), float(bc_x)
        self.device = int(device)
        self.Ndof = self.Nt * self.Nx * 2
        self.Ntot = self.Ndof
        self.Ngauge = 2 * self.Nt * self.Nx
        p = A.WilParams(self.Nt, self.Nx, self.m0, self.beta, self.bc_t, self.bc_x, self.device)
        h = C.c_void_p()
        A.check(A.lib().wil_ctx_create(C.byref(p), C.byref(h)))
        self._h = h
        self._theta = None

    @classmethod
    def from_parameters(cls, p, device=0):
        return cls(p["Nt"], p["Nx"], p["m0"], p["beta"], p["time_boundary_sign"],
                   p["space_boundary_sign"], device)

    def _raise(self, st):
        raise RuntimeError(A.lib().dwf_last_error(self._h).decode() or A.status_string(st))

    def solve_CGNR(self, theta, source, tolerance, max_iterations, solver=A.SOLVER_CG64):
        """dict(x, iterations, normal_residual, dirac_residual)."""
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        self._theta = None
        src = np.ascontiguousarray(source, dtype=np.complex128)
        x = np.empty(self.Ndof, np.complex128)
        info = np.zeros(3)
        st = A.lib().wil_solve_cgnr(self._h, _ptr(th), _ptr(src), float(tolerance),
                                    int(max_iterations), int(solver), _ptr(x), _ptr(info))
        if st != A.DWF_OK:
            self._raise(st)
        return dict(x=x, iterations=int(info[0]), normal_residual=info[1],
                    dirac_residual=info[2])

    def solve_DDdag(self, theta, phi, tolerance, max_iterations, solver=A.SOLVER_CG64):
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        self._theta = None
        ph = np.ascontiguousarray(phi, dtype=np.complex128)
        eta = np.empty(self.Ndof, np.complex128)
        res = C.c_double()
        st = A.lib().wil_solve_dddag(self._h, _ptr(th), _ptr(ph), float(tolerance),
                                     int(max_iterations), int(solver), _ptr(eta), C.byref(res))
        if st != A.DWF_OK:
            self._raise(st)
        return eta

    def hmc_step(self, theta_old, mom, chi, u, epsilon, steps, tolerance, max_iterations,
                 solver=A.SOLVER_CG64):
        """(theta, info) with info['accepted'], ['dH'], ['acceptance_probability']."""
        th = np.ascontiguousarray(theta_old, dtype=np.float64).reshape(-1)
        self._theta = None
        mo = np.ascontiguousarray(mom, dtype=np.float64)
        ch = np.ascontiguousarray(chi, dtype=np.complex128)
        out = np.empty(self.Ngauge)
        hp = A.HmcParams(float(epsilon), int(steps), float(tolerance), int(max_iterations),
                         int(solver))
        info = A.TrajInfo()
        st = A.lib().wil_hmc_step(self._h, C.byref(hp), _ptr(th), _ptr(mo), _ptr(ch), float(u),
                                  _ptr(out), C.byref(info))
        if st != A.DWF_OK:
            self._raise(st)
        return out, info.as_dict()

    def pseudoscalar_correlator(self, thetas, source_t, source_x, tolerance, max_iterations,
                                solver=A.SOLVER_CG64):
        """C(t) per configuration [nconf, Nt] (wilson/include/correlator.hpp:10-40)."""
        th = np.ascontiguousarray(thetas, dtype=np.float64).reshape(-1, self.Ngauge)
        self._theta = None
        nconf = th.shape[0]
        corr = np.zeros((nconf, self.Nt))
        infos = (A.SolveInfo * (2 * nconf))()
        st = A.lib().wil_pseudoscalar_correlator(self._h, nconf, _ptr(th), int(source_t),
                                                 int(source_x), float(tolerance),
                                                 int(max_iterations), int(solver), _ptr(corr),
                                                 infos)
        if st != A.DWF_OK:
            self._raise(st)
        return corr
