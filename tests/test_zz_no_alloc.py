"""dwf_cg_noalloc: the solve for callers that cannot allocate device memory
(code recording a CUDA graph on another thread, plugins confined to their
host's memory pool, allocator-free latency loops). It takes only buffers the
caller already owns and keeps its own in a fixed static device array, so it
is checked here against the context-based dwf_cg on the same inputs, for two
calls in a row (the second reuses the array the first left behind)."""
import ctypes as C

import numpy as np
import pytest

from conftest import random_field, random_theta, rel

pytestmark = pytest.mark.gpu


def _noalloc(A, params, op, theta_t, b_t, x_t, rtol, maxiter, has_guess=0):
    info = A.SolveInfo()
    st = A.lib().dwf_cg_noalloc(C.byref(params), op, C.c_void_p(theta_t.data_ptr()),
                                C.c_void_p(b_t.data_ptr()), C.c_void_p(x_t.data_ptr()),
                                has_guess, float(rtol), int(maxiter), None, C.byref(info))
    return st, info


def test_noalloc_matches_context_solver_twice():
    torch = pytest.importorskip("torch")
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import _capi as A

    rng = np.random.default_rng(99)
    Nt, Nx, Ls, M5, mf = 16, 12, 8, 1.0, 0.1
    d = T.DomainWall(Nt, Nx, Ls, M5, mf)
    params = A.DwfParams(Nt, Nx, Ls, M5, mf, 0.0, 0)
    theta = random_theta(rng, Nt, Nx)
    theta_t = torch.from_numpy(theta.copy()).cuda()
    for call, op in enumerate((T.OP_DDAGD, T.OP_DDDAG)):
        b = random_field(rng, d.Ndof)
        ref = d.conjugate_gradient(op, theta, b, rtol=1e-12, maxiter=4000)
        b_t = torch.from_numpy(b.view(np.float64).copy()).cuda()
        x_t = torch.full_like(b_t, float("nan"))  # stale contents must not matter
        st, info = _noalloc(A, params, op, theta_t, b_t, x_t, 1e-12, 4000)
        torch.cuda.synchronize()
        assert st == A.DWF_OK, f"call {call}: status {st}"
        x = x_t.cpu().numpy().view(np.complex128)
        assert info.converged and info.iterations == ref.iterations
        assert rel(x, ref.x) < 1e-12, f"call {call}"
        assert info.true_relres < 1e-11


def test_noalloc_rejects_lattices_beyond_its_array():
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200 import _capi as A

    big = A.DwfParams(128, 128, 8, 1.0, 0.1, 0.0, 0)  # 131072 sites > DWF_NOALLOC_MAX_SITES
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    st, _ = _noalloc(A, big, 3, t, t, t, 1e-10, 10)
    assert st == A.DWF_BAD_ARG
