"""Host-side mirror of the reference's domain-wall entry points over the C ABI.

Names, argument meaning and error behaviour follow the reference headers:
    apply_D, apply_D_dagger, apply_DD_dagger, apply_D_dagger_D
        (domain_wall/include/dwf_operator.hpp:15-181)
    conjugate_gradient -> CgResult(x, iterations, relative_residual, converged)
        (domain_wall/include/cg_solver.hpp:9-64; raises "CG encountered a zero
         denominator" where the reference throws, :45-46)
Fields are numpy complex128 arrays in the reference layout
((s*Nt + t)*Nx + x)*2 + spin; theta is float64 (mu*Nt + t)*Nx + x.
Device entry points (suffix _dev) take torch CUDA tensors.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi as A
from .learned import LearnedMixin


@dataclass
class CgResult:
    x: np.ndarray
    iterations: int
    relative_residual: float
    converged: bool
    info: dict = field(default_factory=dict)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class DomainWall(LearnedMixin):
    """One device context for a domain-wall lattice (dwf.Nt, dwf.Nx, dwf.N5,
    dwf.M5, dwf.mf, dwf.beta)."""

    def __init__(self, Nt, Nx, Ls, M5, mf, beta=0.0, device=0):
        self.Nt, self.Nx, self.Ls = int(Nt), int(Nx), int(Ls)
        self.M5, self.mf, self.beta = float(M5), float(mf), float(beta)
        self.device = int(device)
        self.Ndof = self.Ls * self.Nt * self.Nx * 2
        self.Ngauge = 2 * self.Nt * self.Nx
        p = A.DwfParams(self.Nt, self.Nx, self.Ls, self.M5, self.mf, self.beta, self.device)
        h = C.c_void_p()
        A.check(A.lib().dwf_ctx_create(C.byref(p), C.byref(h)))
        self._h = h
        self._theta = None

    @classmethod
    def from_parameters(cls, p, device=0):
        return cls(p["Nt"], p["Nx"], p["N5"], p["M5"], p["mf"], p["beta"], device)

    def close(self):
        if getattr(self, "_h", None):
            A.lib().dwf_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def _check(self, st):
        A.check(st, self._h)

    # ---- gauge ---------------------------------------------------------------
    def set_gauge(self, thetas):
        th = np.ascontiguousarray(thetas, dtype=np.float64)
        n = th.size // self.Ngauge
        if n * self.Ngauge != th.size or n < 1:
            raise ValueError("theta size is not a multiple of 2*Nt*Nx")
        self._check(A.lib().dwf_set_gauge(self._h, n, _ptr(th)))
        self._theta = th.reshape(n, self.Ngauge).copy() if n == 1 else None

    def _ensure(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        if th.size != self.Ngauge:
            raise ValueError("theta must hold 2*Nt*Nx link angles")
        if self._theta is None or not np.array_equal(self._theta[0], th):
            self.set_gauge(th)

    # ---- operators (reference names) ------------------------------------------
    def apply(self, op, theta, psi):
        self._ensure(theta)
        v = np.ascontiguousarray(psi, dtype=np.complex128)
        nrhs = v.size // self.Ndof
        if nrhs * self.Ndof != v.size:
            raise ValueError("field size is not a multiple of Ndof")
        out = np.empty_like(v)
        self._check(A.lib().dwf_apply(self._h, op, 0, _ptr(v), _ptr(out), nrhs))
        return out

    def apply_D(self, theta, psi):
        return self.apply(A.OP_D, theta, psi)

    def apply_D_dagger(self, theta, psi):
        return self.apply(A.OP_DDAG, theta, psi)

    def apply_DD_dagger(self, theta, psi):
        return self.apply(A.OP_DDDAG, theta, psi)

    def apply_D_dagger_D(self, theta, psi):
        return self.apply(A.OP_DDAGD, theta, psi)

    def conjugate_gradient(self, op, theta, b, initial_guess=None, rtol=1e-10, maxiter=1000,
                           solver=A.SOLVER_CG64):
        """CG on op in {OP_DDDAG, OP_DDAGD}; mirrors cg_solver.hpp:17-64."""
        self._ensure(theta)
        bb = np.ascontiguousarray(b, dtype=np.complex128)
        if bb.size != self.Ndof:
            raise ValueError("b must hold Ndof complex entries")
        if initial_guess is not None:
            x = np.array(initial_guess, dtype=np.complex128, copy=True).reshape(-1)
        else:
            x = np.zeros(self.Ndof, np.complex128)
        info = A.SolveInfo()
        st = A.lib().dwf_cg(self._h, op, 0, _ptr(bb), _ptr(x), int(initial_guess is not None),
                            float(rtol), int(maxiter), int(solver), C.byref(info))
        if st == A.DWF_ZERO_DENOM:
            raise RuntimeError("CG encountered a zero denominator")
        if st not in (A.DWF_OK, A.DWF_NOT_CONVERGED):
            self._check(st)
        return CgResult(x, info.iterations, info.relres, bool(info.converged), info.as_dict())

    # ---- device entry points (torch tensors) -----------------------------------------
    def _ordered(self):
        """Context manager: the library's stream waits for the work already
        queued on torch's current stream (the tensors' producers), and torch's
        current stream waits for the library's work before anything reads the
        results."""
        import contextlib
        import torch

        @contextlib.contextmanager
        def cm():
            cur = torch.cuda.current_stream()
            ext = torch.cuda.ExternalStream(self.stream_ptr())
            e0 = torch.cuda.Event()
            e0.record(cur)
            ext.wait_event(e0)
            try:
                yield
            finally:
                e1 = torch.cuda.Event()
                e1.record(ext)
                cur.wait_event(e1)
        return cm()

    def _dev_fields(self, t, what):
        """(precision, nrhs) of a contiguous CUDA tensor holding whole fields.
        float64/complex128 -> FP64, float32/complex64 -> FP32; the byte count
        must be an exact multiple of one field."""
        import torch
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError(f"{what}: expected a contiguous CUDA tensor")
        if t.dtype in (torch.float64, torch.complex128):
            prec, csize = 64, 16
        elif t.dtype in (torch.float32, torch.complex64):
            prec, csize = 32, 8
        else:
            raise ValueError(f"{what}: unsupported dtype {t.dtype}")
        nbytes = t.numel() * t.element_size()
        per = self.Ndof * csize
        if nbytes == 0 or nbytes % per:
            raise ValueError(f"{what}: {nbytes} bytes is not a whole number of fields")
        return prec, nbytes // per

    def set_gauge_dev(self, thetas):
        import torch
        if not thetas.is_cuda or thetas.dtype != torch.float64 or not thetas.is_contiguous():
            raise ValueError("thetas: expected a contiguous CUDA float64 tensor")
        n = thetas.numel() // self.Ngauge
        if n < 1 or n * self.Ngauge != thetas.numel():
            raise ValueError("thetas: size is not a multiple of 2*Nt*Nx")
        with self._ordered():
            self._check(A.lib().dwf_set_gauge_dev(self._h, n, C.c_void_p(thetas.data_ptr())))
        self._theta = None

    def apply_dev(self, op, inp, out, conf=0):
        prec, nrhs = self._dev_fields(inp, "in")
        prec2, nrhs2 = self._dev_fields(out, "out")
        if (prec, nrhs) != (prec2, nrhs2):
            raise ValueError("in/out: precision or field count differ")
        with self._ordered():
            self._check(A.lib().dwf_apply_dev(self._h, op, conf, C.c_void_p(inp.data_ptr()),
                                              C.c_void_p(out.data_ptr()), nrhs, prec))

    def cg_batch_dev(self, op, b, x, rhs_conf=None, has_guess=False, rtol=1e-10, maxiter=1000,
                     solver=A.SOLVER_CG64):
        prec, nrhs = self._dev_fields(b, "b")
        prec2, nrhs2 = self._dev_fields(x, "x")
        if prec != 64 or prec2 != 64 or nrhs2 != nrhs:
            raise ValueError("b/x: expected FP64 fields of equal count")
        infos = (A.SolveInfo * nrhs)()
        conf = None
        if rhs_conf is not None:
            conf = np.ascontiguousarray(rhs_conf, dtype=np.int32).reshape(-1)
            if conf.size != nrhs:
                raise ValueError(f"rhs_conf: {conf.size} entries for {nrhs} right-hand sides")
        with self._ordered():
            self._check(A.lib().dwf_cg_batch_dev(
                self._h, op, nrhs, _ptr(conf) if conf is not None else None,
                C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), int(has_guess),
                float(rtol), int(maxiter), int(solver), infos))
        return [i.as_dict() for i in infos]

    def propagators(self, src, rhs_conf=None, rtol=1e-10, maxiter=10000, solver=A.SOLVER_MIXED):
        """x = (D^dag D)^-1 D^dag src for every source (host arrays), as the
        analyzers' propagator solves (correlator.hpp:77-79, :139-142, :213-220)."""
        s = np.ascontiguousarray(src, dtype=np.complex128)
        nrhs = s.size // self.Ndof
        if nrhs < 1 or nrhs * self.Ndof != s.size:
            raise ValueError("src: not a whole number of fields")
        x = np.empty_like(s)
        infos = (A.SolveInfo * nrhs)()
        conf = None
        if rhs_conf is not None:
            conf = np.ascontiguousarray(rhs_conf, dtype=np.int32).reshape(-1)
            if conf.size != nrhs:
                raise ValueError("rhs_conf: wrong length")
        self._check(A.lib().dwf_propagators(self._h, nrhs, _ptr(conf) if conf is not None else None,
                                            _ptr(s), _ptr(x), float(rtol), int(maxiter),
                                            int(solver), infos))
        return x, [i.as_dict() for i in infos]

    def propagators_dev(self, src, x, rhs_conf=None, rtol=1e-10, maxiter=10000,
                        solver=A.SOLVER_MIXED):
        prec, nrhs = self._dev_fields(src, "src")
        prec2, nrhs2 = self._dev_fields(x, "x")
        if prec != 64 or prec2 != 64 or nrhs2 != nrhs:
            raise ValueError("src/x: expected FP64 fields of equal count")
        infos = (A.SolveInfo * nrhs)()
        conf = None
        if rhs_conf is not None:
            conf = np.ascontiguousarray(rhs_conf, dtype=np.int32).reshape(-1)
            if conf.size != nrhs:
                raise ValueError("rhs_conf: wrong length")
        with self._ordered():
            self._check(A.lib().dwf_propagators_dev(
                self._h, nrhs, _ptr(conf) if conf is not None else None,
                C.c_void_p(src.data_ptr()), C.c_void_p(x.data_ptr()), float(rtol), int(maxiter),
                int(solver), infos))
        return [i.as_dict() for i in infos]

    # ---- HMC pieces (reference names) -----------------------------------------------
    def gauge_action_force(self, theta):
        """(action, force) -- domain_wall/include/gauge.hpp:26-62."""
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        self._theta = None
        a = C.c_double()
        f = np.empty(self.Ngauge)
        self._check(A.lib().dwf_gauge_action_force(self._h, _ptr(th), C.byref(a), _ptr(f)))
        return a.value, f

    def average_plaquette(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        self._theta = None
        p = C.c_double()
        self._check(A.lib().dwf_average_plaquette(self._h, _ptr(th), C.byref(p)))
        return p.value

    def pseudofermion_action_force(self, theta, phi, eta_guess=None, rtol=1e-10, maxiter=1000,
                                   solver=A.SOLVER_CG64):
        """dict(action, force, eta, iterations, relative_residual) --
        domain_wall/include/pseudofermion.hpp:22-166 (raises where it throws)."""
        th = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        self._theta = None
        ph = np.ascontiguousarray(phi, dtype=np.complex128)
        g = np.ascontiguousarray(eta_guess, dtype=np.complex128) if eta_guess is not None else None
        a = C.c_double()
        f = np.empty(self.Ngauge)
        eta = np.empty(self.Ndof, np.complex128)
        info = A.SolveInfo()
        st = A.lib().dwf_pf_action_force(self._h, _ptr(th), _ptr(ph),
                                          _ptr(g) if g is not None else None, float(rtol),
                                          int(maxiter), int(solver), C.byref(a), _ptr(f),
                                          _ptr(eta), C.byref(info))
        if st != A.DWF_OK:
            raise RuntimeError(A.lib().dwf_last_error(self._h).decode() or A.status_string(st))
        return dict(action=a.value, force=f, eta=eta, iterations=info.iterations,
                    relative_residual=info.relres, info=info.as_dict())

    def hmc_trajectory(self, theta0, chi, mom, epsilon, steps, rtol=1e-10, maxiter=1000,
                       solver=A.SOLVER_CG64):
        """Proposal and trajectory report for one domain-wall trajectory
        (domain_wall/generate_configs.cpp:56-160); Metropolis is the caller's."""
        th = np.ascontiguousarray(theta0, dtype=np.float64).reshape(-1)
        self._theta = None
        ch = np.ascontiguousarray(chi, dtype=np.complex128)
        mo = np.ascontiguousarray(mom, dtype=np.float64)
        out = np.empty(self.Ngauge)
        hp = A.HmcParams(float(epsilon), int(steps), float(rtol), int(maxiter), int(solver))
        info = A.TrajInfo()
        st = A.lib().dwf_hmc_trajectory(self._h, C.byref(hp), _ptr(th), _ptr(ch), _ptr(mo),
                                         _ptr(out), C.byref(info))
        if st != A.DWF_OK:
            raise RuntimeError(A.lib().dwf_last_error(self._h).decode() or A.status_string(st))
        return out, info.as_dict()

    # ---- measurements ---------------------------------------------------------------
    def measure(self, thetas, z4=None, n_point_times=2, n_wall_times=2, n_noise=0,
                max_momentum=0, rtol=1e-8, maxiter=800, solver=A.SOLVER_MIXED):
        """Batched propagators and contractions for every configuration
        (domain_wall/include/correlator.hpp:27-310). Returns dict of
        cpp, cj5 [nconf, Nt], loop [nconf, Nt*Nx] complex, mom_cpp
        [nconf, max_momentum+1, Nt] and the per-right-hand-side solve reports."""
        th = np.ascontiguousarray(thetas, dtype=np.float64).reshape(-1, self.Ngauge)
        nconf = th.shape[0]
        self._theta = None
        V = self.Nt * self.Nx
        zz = None
        if n_noise > 0:
            zz = np.ascontiguousarray(z4, dtype=np.int8).reshape(-1)
            if zz.size != nconf * n_noise * V * 2:
                raise ValueError("z4: expected nconf*n_noise*Nt*Nx*2 digits")
        mp = A.MeasureParams(int(n_point_times), int(n_wall_times), int(n_noise),
                             int(max_momentum), float(rtol), int(maxiter), int(solver))
        cpp = np.zeros((nconf, self.Nt))
        cj5 = np.zeros((nconf, self.Nt))
        loop = np.zeros((nconf, V), np.complex128)
        nmom = max_momentum + 1 if n_point_times > 0 else 0
        mom = np.zeros((nconf, max(nmom, 1), self.Nt))
        R = 2 * n_point_times + 2 * n_wall_times + n_noise
        infos = (A.SolveInfo * (nconf * R))()
        st = A.lib().dwf_measure(self._h, C.byref(mp), nconf, _ptr(th),
                                 _ptr(zz) if zz is not None else None, _ptr(cpp), _ptr(cj5),
                                 _ptr(loop), _ptr(mom), infos)
        if st != A.DWF_OK:
            raise RuntimeError(A.lib().dwf_last_error(self._h).decode() or A.status_string(st))
        return dict(cpp=cpp, cj5=cj5, loop=loop, mom_cpp=mom[:, :nmom],
                    info=[i.as_dict() for i in infos])

    def set_eo_kernel(self, kernel):
        """Even-odd solve kernel: -1 automatic (cluster kernel where it fits), 0 grid-wide."""
        self._check(A.lib().dwf_set_eo_kernel(self._h, int(kernel)))

    def set_dslash_variant(self, variant, chunk=None):
        """Force a Dslash kernel for apply/apply_dev (0 site, 1 column, 2 site
        with shuffled x neighbours, 3 t sweep, 4 Wilson rows, 5 column with
        shuffled x neighbours; -1 autotune, the default), and optionally the t
        sweep's chunk length in rows (0: automatic and tuned)."""
        self._check(A.lib().dwf_set_dslash_variant(self._h, int(variant)))
        if chunk is not None:
            self._check(A.lib().dwf_set_dslash_chunk(self._h, int(chunk)))

    def dslash_variant(self, precision, nrhs):
        """The Dslash kernel the autotuner chose for a precision (64 or 32) and
        batch size (-1 before the first application of that kind)."""
        return int(A.lib().dwf_dslash_variant(self._h, int(precision), int(nrhs)))

    def launch_count(self):
        return int(A.lib().dwf_launch_count(self._h))

    def solver_kernel_ms(self, kind=0):
        """(ms, launches) of the persistent solver kernels of one kind:
        0 full lattice, 1 even-odd (either kernel), 2 even-odd cluster kernel."""
        n = C.c_uint64()
        ms = A.lib().dwf_solver_kernel_ms(self._h, int(kind), C.byref(n))
        return ms, n.value

    def graph_replays(self):
        """(replays so far, graphs cached) of the captured even-odd propagator
        chunks."""
        n = C.c_int()
        r = A.lib().dwf_graph_replays(self._h, C.byref(n))
        return int(r), n.value

    def sync(self):
        self._check(A.lib().dwf_sync(self._h))

    def stream_ptr(self):
        return A.lib().dwf_stream(self._h)
