"""dwf_cg_noalloc: the solve for callers that cannot allocate device memory
(code that runs while another thread records a CUDA graph, plugins confined to
their host's memory pool, allocator-free latency loops). It takes only buffers
the caller already owns and keeps its own in a fixed static device array, so it
is checked here against the context-based dwf_cg on the same inputs: for two
calls in a row (the second reuses the array the first left behind), from a warm
start, on a caller's stream, with the device's free memory unchanged across a
call, and while another thread holds a (thread-local mode) graph capture open."""
import ctypes as C
import threading

import numpy as np
import pytest

from conftest import random_field, random_theta, rel

pytestmark = pytest.mark.gpu

Nt, Nx, Ls, M5, mf = 16, 12, 8, 1.0, 0.1


def _noalloc(A, params, op, theta_t, b_t, x_t, rtol, maxiter, has_guess=0, stream=None):
    info = A.SolveInfo()
    st = A.lib().dwf_cg_noalloc(C.byref(params), op, C.c_void_p(theta_t.data_ptr()),
                                C.c_void_p(b_t.data_ptr()), C.c_void_p(x_t.data_ptr()),
                                has_guess, float(rtol), int(maxiter),
                                C.c_void_p(stream) if stream else None, C.byref(info))
    return st, info


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    import three_part_dwf_study_b200 as T
    from three_part_dwf_study_b200 import _capi as A

    rng = np.random.default_rng(99)
    d = T.DomainWall(Nt, Nx, Ls, M5, mf)
    params = A.DwfParams(Nt, Nx, Ls, M5, mf, 0.0, 0)
    theta = random_theta(rng, Nt, Nx)
    theta_t = torch.from_numpy(theta.copy()).cuda()
    yield torch, T, A, rng, d, params, theta, theta_t
    d.close()


def _dev(torch, z):
    return torch.from_numpy(np.ascontiguousarray(z).view(np.float64).copy()).cuda()


def _host(x_t):
    return x_t.cpu().numpy().view(np.complex128)


def test_noalloc_matches_context_solver_twice(setup):
    torch, T, A, rng, d, params, theta, theta_t = setup
    for call, op in enumerate((T.OP_DDAGD, T.OP_DDDAG)):
        b = random_field(rng, d.Ndof)
        ref = d.conjugate_gradient(op, theta, b, rtol=1e-12, maxiter=4000)
        b_t = _dev(torch, b)
        x_t = torch.full_like(b_t, float("nan"))  # stale contents must not matter
        st, info = _noalloc(A, params, op, theta_t, b_t, x_t, 1e-12, 4000)
        torch.cuda.synchronize()
        assert st == A.DWF_OK, f"call {call}: status {st}"
        assert info.converged and info.iterations == ref.iterations
        assert rel(_host(x_t), ref.x) < 1e-12, f"call {call}"
        assert info.true_relres < 1e-11


def test_noalloc_warm_start_on_a_caller_stream(setup):
    """has_guess = 1 reads x as the starting point (the reference's
    initial_guess): same iterations and answer as dwf_cg from that guess, fewer
    iterations than from zero; the work runs on the caller's stream."""
    torch, T, A, rng, d, params, theta, theta_t = setup
    op = T.OP_DDAGD
    b = random_field(rng, d.Ndof)
    cold = d.conjugate_gradient(op, theta, b, rtol=1e-12, maxiter=4000)
    guess = cold.x + 1e-4 * random_field(rng, d.Ndof) * np.abs(cold.x).mean()
    ref = d.conjugate_gradient(op, theta, b, initial_guess=guess, rtol=1e-12, maxiter=4000)
    stream = torch.cuda.Stream()
    b_t, x_t = _dev(torch, b), _dev(torch, guess)
    torch.cuda.synchronize()
    st, info = _noalloc(A, params, op, theta_t, b_t, x_t, 1e-12, 4000, has_guess=1,
                        stream=stream.cuda_stream)
    stream.synchronize()
    assert st == A.DWF_OK
    assert info.iterations == ref.iterations < cold.iterations
    assert rel(_host(x_t), ref.x) < 1e-12
    assert rel(_host(x_t), cold.x) < 1e-9


def test_noalloc_leaves_device_memory_unchanged(setup):
    """After the first call (which loads the module and so its static array),
    a call changes the device's free memory by zero bytes."""
    torch, T, A, rng, d, params, theta, theta_t = setup
    b_t = _dev(torch, random_field(rng, d.Ndof))
    x_t = torch.empty_like(b_t)
    st, _ = _noalloc(A, params, T.OP_DDAGD, theta_t, b_t, x_t, 1e-10, 4000)
    assert st == A.DWF_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st, info = _noalloc(A, params, T.OP_DDAGD, theta_t, b_t, x_t, 1e-10, 4000)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert st == A.DWF_OK and info.converged
    assert free1 == free0


def test_noalloc_while_another_thread_captures(setup):
    """One thread holds a CUDA graph capture open (torch.cuda.graph in
    thread-local capture mode, as the entry point's documentation requires of
    a concurrent capture) while another runs the solve on its own stream: both
    the solve and the captured graph succeed. Every tensor is allocated before
    the capture."""
    torch, T, A, rng, d, params, theta, theta_t = setup
    op = T.OP_DDAGD
    b = random_field(rng, d.Ndof)
    ref = d.conjugate_gradient(op, theta, b, rtol=1e-12, maxiter=4000)
    b_t = _dev(torch, b)
    x_t = torch.empty_like(b_t)
    src = torch.arange(4096, dtype=torch.float32, device="cuda")
    dst = torch.zeros_like(src)
    solve_stream, cap_stream = torch.cuda.Stream(), torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    capturing, solved = threading.Event(), threading.Event()
    out = {}

    def solve():
        try:
            if capturing.wait(60):
                out["st"], out["info"] = _noalloc(A, params, op, theta_t, b_t, x_t, 1e-12,
                                                  4000, stream=solve_stream.cuda_stream)
        finally:
            solved.set()

    worker = threading.Thread(target=solve)
    worker.start()
    torch.cuda.synchronize()
    try:
        with torch.cuda.graph(graph, stream=cap_stream, capture_error_mode="thread_local"):
            dst.copy_(src)
            dst.mul_(2.0)
            capturing.set()
            assert solved.wait(120)
    finally:
        capturing.set()
        worker.join(120)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(dst, 2.0 * src)
    assert out.get("st") == A.DWF_OK
    assert out["info"].iterations == ref.iterations
    assert rel(_host(x_t), ref.x) < 1e-12


def test_noalloc_rejects_lattices_beyond_its_array(setup):
    torch, T, A, rng, d, params, theta, theta_t = setup
    big = A.DwfParams(128, 128, 8, 1.0, 0.1, 0.0, 0)  # 131072 sites > DWF_NOALLOC_MAX_SITES
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    st, _ = _noalloc(A, big, 3, t, t, t, 1e-10, 10)
    assert st == A.DWF_BAD_ARG
