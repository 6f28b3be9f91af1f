"""Even-odd (Schur-complement) preconditioned propagator solves on the GPU.

The even-odd stage solves Dhat x_o = b_o - H_oe M5^-1 b_e on the odd sites and
reconstructs x_e; the full-lattice FP64 solve that follows enforces the
reference's stopping rule on D^dag D. Checked: the stage does nearly all the
work (the full-lattice check needs a few iterations at most), the
result equals the FP64 reference-algorithm solution, the analyzer outputs
match the reference's golden vectors, and lattices the stage cannot take fall
back."""
import numpy as np
import pytest

from conftest import random_theta, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import three_part_dwf_study_b200 as T
    return T


def boundary_sources(rng, Nt, Nx, Ls, n):
    srcs = np.zeros((n, Ls, Nt, Nx, 2), np.complex128)
    for k in range(n):
        eta = np.exp(0.5j * np.pi * rng.integers(0, 4, size=(Nt, Nx, 2)))
        srcs[k, 0, :, :, 1] = eta[:, :, 1]
        srcs[k, Ls - 1, :, :, 0] = eta[:, :, 0]
    return srcs.reshape(n, -1)


@pytest.mark.parametrize("shape,mf", [((16, 12, 8), 0.1), ((32, 32, 16), 0.05),
                                      ((8, 6, 1), 0.3)])
def test_eo_propagators_match_fp64_reference(T, shape, mf):
    Nt, Nx, Ls = shape
    rng = np.random.default_rng(Nt + Nx + Ls)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, mf)
    th = random_theta(rng, Nt, Nx)
    d.set_gauge(th)
    src = boundary_sources(rng, Nt, Nx, Ls, 3)
    x_eo, info_eo = d.propagators(src, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    x_64, info_64 = d.propagators(src, rtol=1e-12, maxiter=20000, solver=T.SOLVER_CG64)
    for k in range(3):
        e, f = info_eo[k], info_64[k]
        assert e["converged"] and e["true_relres"] <= 1e-10
        assert e["schur_iterations"] > 0
        # the even-odd stage did the work: the full-lattice check needs a few
        # of its (warm-start) reliable-update periods at most
        assert e["iterations"] - e["schur_iterations"] <= max(32, e["schur_iterations"] // 4)
        assert e["schur_iterations"] < f["iterations"]
        assert rel(x_eo[k], x_64[k]) < 1e-7


def test_eo_measure_matches_reference_golden(T, golden):
    from three_part_dwf_study_b200.rng import z4_digits
    g = golden("dwf_8x8x4")
    p = g.p
    d = T.DomainWall(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"])
    nn = p["eta.noise_vectors"]
    z4 = z4_digits(p["eta.random_seed"], nn * d.Nt * d.Nx * 2)
    m = d.measure(g.npy("in_theta.npy"), z4=z4, n_point_times=2, n_wall_times=2, n_noise=nn,
                  max_momentum=p["analysis.max_momentum"], rtol=1e-12, maxiter=4000,
                  solver=T.SOLVER_EO_MIXED)
    assert rel(m["cpp"][0], g.npy("out_cpp.npy")) < 1e-9
    assert rel(m["cj5"][0], g.npy("out_cj5.npy")) < 1e-9
    assert rel(m["mom_cpp"][0], g.npy("out_mom.npy")) < 1e-9
    assert rel(m["loop"][0], g.field("out_loop.npy")) < 1e-9
    assert all(i["schur_iterations"] > 0 for i in m["info"])


def test_eo_falls_back_on_odd_lattices(T):
    rng = np.random.default_rng(9)
    Nt, Nx, Ls = 7, 6, 4
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.1)
    d.set_gauge(random_theta(rng, Nt, Nx))
    src = boundary_sources(rng, Nt, Nx, Ls, 2)
    x, info = d.propagators(src, rtol=1e-10, maxiter=5000, solver=T.SOLVER_EO_MIXED)
    assert all(i["converged"] and i["true_relres"] <= 1e-10 and i["schur_iterations"] == 0
               for i in info)


def test_eo_phase_timers(T):
    """The even-odd kernel's optional phase timers count one entry per Schur
    iteration for each operator phase, and cost nothing when off."""
    import ctypes as C
    from three_part_dwf_study_b200 import _capi as A
    rng = np.random.default_rng(3)
    d = T.DomainWall(16, 12, 8, 1.0, 0.1)
    d.set_gauge(random_theta(rng, 16, 12))
    src = boundary_sources(rng, 16, 12, 8, 2)
    ms = (C.c_double * 8)()
    cnt = (C.c_uint64 * 8)()
    assert A.lib().dwf_eo_phase_times(d.handle, ms, cnt) == A.DWF_BAD_ARG  # off by default
    assert A.lib().dwf_eo_phase_profile(d.handle, 1) == 0
    _, info = d.propagators(src, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    assert A.lib().dwf_eo_phase_times(d.handle, ms, cnt) == 0
    it = max(i["schur_iterations"] for i in info)
    assert cnt[0] == cnt[1] == cnt[3] == cnt[4] == it
    assert all(ms[k] > 0.0 for k in (0, 1, 3, 4))
    assert A.lib().dwf_eo_phase_profile(d.handle, 0) == 0
    d.close()


@pytest.mark.parametrize("shape,nrhs", [((64, 64, 16), 6), ((64, 32, 16), 20), ((32, 16, 24), 3)])
def test_cluster_kernel_matches_grid_kernel(T, shape, nrhs):
    """The even-odd solve on one thread-block cluster per right-hand side (FP32
    fields in distributed shared memory; cluster of 16 CTAs at 64x64x16, of 8 at
    64x32x16, Ls = 24 with six slices per lane at 32x16x24) against the
    grid-wide kernel on the same sources: both meet the FP64 true residual, the
    solutions agree to the solvers' accuracy and the Schur iteration counts
    agree closely (more right-hand sides than clusters at 64x32x16, so
    clusters take several right-hand sides in turn)."""
    Nt, Nx, Ls = shape
    rng = np.random.default_rng(Nt * Nx + Ls)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.05)
    from three_part_dwf_study_b200.ensemble import quenched_theta
    d.set_gauge(quenched_theta(rng, Nt, Nx, 3.0))
    src = boundary_sources(rng, Nt, Nx, Ls, nrhs)
    n0 = d.solver_kernel_ms(2)[1]
    x_cl, info_cl = d.propagators(src, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    assert d.solver_kernel_ms(2)[1] == n0 + 1  # the cluster kernel ran
    d.set_eo_kernel(0)
    x_gr, info_gr = d.propagators(src, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    d.set_eo_kernel(-1)
    for k in range(nrhs):
        c, g = info_cl[k], info_gr[k]
        assert c["converged"] and c["true_relres"] <= 1e-10, k
        assert g["converged"] and g["true_relres"] <= 1e-10, k
        assert c["schur_iterations"] > 0
        assert abs(c["schur_iterations"] - g["schur_iterations"]) <= 0.1 * g["schur_iterations"] + 8
        assert rel(x_cl[k], x_gr[k]) < 1e-7, k
    d.close()


def test_cluster_solve_replays_its_graph(T):
    """The even-odd cluster path runs each chunk (source preparation, the
    solver launch, reconstruction) as a captured CUDA graph: the first call
    captures it, the next calls with the same batch size and buffers replay
    it, a replay with new sources solves those sources (the graph reads the
    buffers, not copies of them), and the replayed results are bit-identical
    to the captured run's for the same input."""
    from three_part_dwf_study_b200.ensemble import quenched_theta
    Nt, Nx, Ls = 32, 32, 16
    rng = np.random.default_rng(3232)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.05)
    d.set_gauge(quenched_theta(rng, Nt, Nx, 3.0))
    src1 = boundary_sources(rng, Nt, Nx, Ls, 5)
    src2 = boundary_sources(rng, Nt, Nx, Ls, 5)
    r0, _ = d.graph_replays()
    n0 = d.solver_kernel_ms(2)[1]
    x1, i1 = d.propagators(src1, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    r1, cached = d.graph_replays()
    assert d.solver_kernel_ms(2)[1] == n0 + 1 and cached >= 1 and r1 == r0
    x1b, i1b = d.propagators(src1, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    assert d.graph_replays()[0] == r1 + 1
    assert np.array_equal(x1, x1b)
    assert [i["schur_iterations"] for i in i1] == [i["schur_iterations"] for i in i1b]
    x2, i2 = d.propagators(src2, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    assert d.graph_replays()[0] == r1 + 2
    # the same sources on the grid-wide kernel (no graph)
    d.set_eo_kernel(0)
    x2g, i2g = d.propagators(src2, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    d.set_eo_kernel(-1)
    for k in range(5):
        for info in (i1[k], i2[k], i2g[k]):
            assert info["converged"] and info["true_relres"] <= 1e-10
        assert rel(x2[k], x2g[k]) < 1e-7, k
    d.close()


def test_host_batch_solves_in_overlapped_chunks(T):
    """dwf_propagators with host buffers and at least two waves of the cluster
    solver runs in chunks of whole waves (here 16 sources at 64x64x16: two
    waves, then a ragged chunk), the copies of one chunk overlapping the solve
    of the other: the solutions and iteration counts equal those of the same
    batch solved on device buffers in one call, page-locked and pageable host
    buffers alike, and a second call replays the chunks' graphs."""
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200.ensemble import quenched_theta
    Nt, Nx, Ls = 64, 64, 16
    rng = np.random.default_rng(6464)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.05)
    d.set_gauge(quenched_theta(rng, Nt, Nx, 3.0))
    src = boundary_sources(rng, Nt, Nx, Ls, 16)
    s_dev = torch.from_numpy(src).cuda()
    x_dev = torch.empty_like(s_dev)
    n0 = d.solver_kernel_ms(2)[1]
    i_dev = d.propagators_dev(s_dev, x_dev, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    assert d.solver_kernel_ms(2)[1] == n0 + 1
    x_ref = x_dev.cpu().numpy()
    n1 = d.solver_kernel_ms(2)[1]
    x_h, i_h = d.propagators(src, rtol=1e-10, maxiter=20000, solver=T.SOLVER_EO_MIXED)
    chunks = d.solver_kernel_ms(2)[1] - n1
    assert 2 <= chunks <= 4
    for k in range(16):
        assert i_h[k]["converged"] and i_h[k]["true_relres"] <= 1e-10, k
        assert i_h[k]["schur_iterations"] == i_dev[k]["schur_iterations"], k
    # each right-hand side is solved as in the single batch unless a batch
    # needed the full-lattice continuation (decided per chunk)
    if all(i["iterations"] == i["schur_iterations"] for i in i_dev):
        assert np.array_equal(x_h, x_ref)
    else:
        assert rel(x_h, x_ref) < 1e-9
    # page-locked host buffers, and the chunk graphs replayed
    r0, _ = d.graph_replays()
    s_pin = torch.from_numpy(src).pin_memory()
    x_pin = torch.empty_like(s_pin).pin_memory()
    infos = (T._capi.SolveInfo * 16)()
    import ctypes as C
    T._capi.check(T._capi.lib().dwf_propagators(d.handle, 16, None, C.c_void_p(s_pin.data_ptr()),
                                                C.c_void_p(x_pin.data_ptr()), 1e-10, 20000,
                                                T.SOLVER_EO_MIXED, infos), d.handle)
    assert d.graph_replays()[0] == r0 + chunks
    assert np.array_equal(x_pin.numpy(), x_h)
    d.close()
