"""Learned preconditioner of the propagator solves (no counterpart in the
reference): a gauge-equivariant parallel-transport convolution network
N ~ D^-1 with four layers (C0 -> hidden -> hidden -> hidden -> C0 complex
channels per 4-D site), trained on the GPU by the library's own forward and
backward kernels, and used by ``SOLVER_LEARNED`` as the right preconditioner of
an FP32 BiCGStab inside FP64 defect correction. See include/dwf_b200.h for the
layer definition and the weight layout."""
import ctypes as C

import numpy as np

from . import _capi as A


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _conf(rhs_conf, n):
    if rhs_conf is None:
        return None
    c = np.ascontiguousarray(rhs_conf, dtype=np.int32).reshape(-1)
    if c.size != n:
        raise ValueError(f"rhs_conf: {c.size} entries for {n} right-hand sides")
    return c


class LearnedMixin:
    """Methods of DomainWall / Wilson for the learned preconditioner."""

    def lp_init(self, hidden=16, seed=1):
        self._check(A.lib().dwf_lp_init(self._h, int(hidden), int(seed)))
        self._lp_hidden = int(hidden)

    def lp_shapes(self):
        """[(cout, cin)] of the four layers."""
        C0 = 2 * (self.Ls if hasattr(self, "Ls") else 1)
        H = self._lp_hidden
        ch = [C0, H, H, H, C0]
        return [(ch[l + 1], ch[l]) for l in range(4)]

    def lp_weights(self):
        """List of four complex64 arrays [9, cout, cin]."""
        n = C.c_long()
        self._check(A.lib().dwf_lp_weights_size(self._h, C.byref(n)))
        w = np.empty(n.value, np.complex64)
        self._check(A.lib().dwf_lp_get_weights(self._h, _ptr(w)))
        out, o = [], 0
        for co, ci in self.lp_shapes():
            k = 9 * co * ci
            out.append(w[o:o + k].reshape(9, co, ci).copy())
            o += k
        return out

    def lp_set_weights(self, ws):
        flat = np.concatenate([np.asarray(w, np.complex64).reshape(-1) for w in ws])
        self._check(A.lib().dwf_lp_set_weights(self._h, _ptr(flat)))

    def lp_transports(self, conf=0):
        T = np.empty(self.Nt * self.Nx * 9, np.complex64)
        self._check(A.lib().dwf_lp_transports(self._h, int(conf), _ptr(T)))
        return T.reshape(self.Nt * self.Nx, 9)

    def lp_apply_dev(self, inp, out, adjoint=False, rhs_conf=None):
        """out = N inp (or N^dag inp): complex64 CUDA tensors of whole fields."""
        prec, nrhs = self._dev_fields(inp, "in")
        prec2, nrhs2 = self._dev_fields(out, "out")
        if prec != 32 or prec2 != 32 or nrhs != nrhs2:
            raise ValueError("in/out: expected FP32 fields of equal count")
        c = _conf(rhs_conf, nrhs)
        with self._ordered():
            self._check(A.lib().dwf_lp_apply_dev(self._h, int(adjoint), nrhs,
                                                 _ptr(c) if c is not None else None,
                                                 C.c_void_p(inp.data_ptr()),
                                                 C.c_void_p(out.data_ptr())))

    def lp_layer_dev(self, layer, inp, out, adjoint=False, rhs_conf=None):
        """One layer on complex64 CUDA tensors [nrhs, V, C] (network layout)."""
        nrhs = inp.shape[0]
        c = _conf(rhs_conf, nrhs)
        with self._ordered():
            self._check(A.lib().dwf_lp_layer_dev(self._h, int(layer), int(adjoint), nrhs,
                                                 _ptr(c) if c is not None else None,
                                                 C.c_void_p(inp.data_ptr()),
                                                 C.c_void_p(out.data_ptr())))

    def lp_loss_grad_dev(self, rho, e, pair_conf=None):
        """(loss, [grad per layer]) on complex64 CUDA tensors of pairs."""
        prec, n = self._dev_fields(rho, "rho")
        c = _conf(pair_conf, n)
        nw = C.c_long()
        self._check(A.lib().dwf_lp_weights_size(self._h, C.byref(nw)))
        g = np.empty(nw.value, np.complex64)
        loss = C.c_double()
        with self._ordered():
            self._check(A.lib().dwf_lp_loss_grad_dev(self._h, n, _ptr(c) if c is not None else None,
                                                     C.c_void_p(rho.data_ptr()),
                                                     C.c_void_p(e.data_ptr()), C.byref(loss),
                                                     _ptr(g)))
        out, o = [], 0
        for co, ci in self.lp_shapes():
            k = 9 * co * ci
            out.append(g[o:o + k].reshape(9, co, ci).copy())
            o += k
        return loss.value, out

    def lp_train(self, steps=1000, batch=8, lr=3e-3, lr_decay_steps=0, pairs_per_conf=16,
                 solver_iters=0, solver_every=2, solver_maxiter=20000, seed=7, history=False):
        """Generate pairs on the uploaded configurations and train with Adam on
        the GPU. Returns the info dict (and the per-step loss if history)."""
        p = A.LpTrainParams(int(steps), int(batch), float(lr), int(lr_decay_steps),
                            int(pairs_per_conf), int(solver_iters), int(solver_every),
                            int(solver_maxiter), int(seed))
        info = A.LpTrainInfo()
        h = np.zeros(max(int(steps), 1)) if history else None
        self._check(A.lib().dwf_lp_train(self._h, C.byref(p), C.byref(info),
                                         _ptr(h) if h is not None else None))
        return (info.as_dict(), h) if history else info.as_dict()

    def lp_time_network(self, nrhs, reps=10):
        """(ms per network application, flops per application) on nrhs fields."""
        ms = C.c_double()
        fl = C.c_double()
        self._check(A.lib().dwf_lp_time_network(self._h, int(nrhs), int(reps), C.byref(ms), C.byref(fl)))
        return ms.value, fl.value

    def lp_set_variant(self, variant):
        """Layer kernel: -1 automatic (the first learned solve per batch size
        times both kernels and keeps the faster), 0 mma.sync, 1 tcgen05."""
        self._check(A.lib().dwf_lp_set_variant(self._h, int(variant)))

    def lp_set_solver(self, inner_tol=3e-4, inner_maxiter=400, outer_max=40):
        self._check(A.lib().dwf_lp_set_solver(self._h, float(inner_tol), int(inner_maxiter),
                                              int(outer_max)))

    def lp_set_krylov(self, method=A.LP_GCR, restart=4):
        """Inner Krylov method of the learned solver: LP_GCR (flexible GCR
        restarted every `restart` iterations, 4/8/12/16) or LP_BICGSTAB."""
        self._check(A.lib().dwf_lp_set_krylov(self._h, int(method), int(restart)))
