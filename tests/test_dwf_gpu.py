"""Domain-wall operator and solver on the GPU, through the C ABI, against the
CPU oracle and the reference's golden vectors.

Tolerances: FP64 operator outputs within 1e-13 relative (different
summation order and FMA contraction only); FP64 CG solutions within 1e-12
relative when both solve to rtol 1e-13; the mixed path is checked by its FP64
true residual."""
import numpy as np
import pytest

from conftest import random_field, random_theta, rel
from oracle import oracle as O

pytestmark = pytest.mark.gpu

OPS = [(0, "D"), (1, "Ddag"), (2, "DDdag"), (3, "DdagD")]


@pytest.fixture(scope="module")
def tdwf():
    import three_part_dwf_study_b200 as T
    return T


@pytest.mark.parametrize("case", ["dwf_8x8x4", "dwf_6x10x3"])
def test_operators_match_golden(tdwf, golden, case):
    g = golden(case)
    p = g.p
    d = tdwf.DomainWall(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"])
    th, psi = g.npy("in_theta.npy"), g.field("in_psi.npy")
    for op, name in OPS:
        assert rel(d.apply(op, th, psi), g.field(f"out_{name}.npy")) < 1e-13, name


@pytest.mark.parametrize("shape", [(8, 8, 4), (6, 10, 3), (16, 12, 8), (3, 5, 1), (2, 2, 2),
                                   (64, 64, 16)])
def test_operators_match_oracle(tdwf, shape):
    Nt, Nx, Ls = shape
    rng = np.random.default_rng(Nt * 1000 + Nx * 10 + Ls)
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.1, 0.07)
    o = O.Dwf(Nt, Nx, Ls, 1.1, 0.07)
    th = random_theta(rng, Nt, Nx)
    psi = random_field(rng, o.ndof)
    for op, name in OPS:
        assert rel(d.apply(op, th, psi), o.apply(op, th, psi)) < 1e-13, name


def test_multi_rhs_apply_and_adjointness(tdwf):
    rng = np.random.default_rng(3)
    Nt, Nx, Ls = 12, 10, 6
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.0, 0.05)
    o = O.Dwf(Nt, Nx, Ls, 1.0, 0.05)
    th = random_theta(rng, Nt, Nx)
    psi = random_field(rng, 3 * o.ndof)
    out = d.apply(0, th, psi).reshape(3, -1)
    for k in range(3):
        assert rel(out[k], o.apply(0, th, psi.reshape(3, -1)[k])) < 1e-13
    a, b = random_field(rng, o.ndof), random_field(rng, o.ndof)
    lhs = np.vdot(a, d.apply(0, th, b))
    rhs = np.vdot(d.apply(1, th, a), b)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_gauge_covariance(tdwf):
    """theta_mu(y) -> theta_mu(y) + a(y) - a(y + mu), psi(y) -> e^{i a(y)} psi(y)
    maps D psi -> e^{i a} D psi (boundary signs are untouched)."""
    rng = np.random.default_rng(4)
    Nt, Nx, Ls = 8, 6, 4
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.0, 0.1)
    th = random_theta(rng, Nt, Nx).reshape(2, Nt, Nx)
    alpha = rng.uniform(-np.pi, np.pi, (Nt, Nx))
    th2 = th.copy()
    th2[0] += alpha - np.roll(alpha, -1, axis=0)
    th2[1] += alpha - np.roll(alpha, -1, axis=1)
    psi = random_field(rng, Ls * Nt * Nx * 2).reshape(Ls, Nt, Nx, 2)
    ph = np.exp(1j * alpha)[None, :, :, None]
    out1 = d.apply(0, th.ravel(), psi.ravel()).reshape(psi.shape)
    out2 = d.apply(0, th2.ravel(), (ph * psi).ravel()).reshape(psi.shape)
    assert rel(out2, ph * out1) < 1e-13


@pytest.mark.parametrize("case", ["dwf_8x8x4", "dwf_6x10x3"])
def test_cg_matches_golden(tdwf, golden, case):
    g = golden(case)
    p = g.p
    d = tdwf.DomainWall(p["dwf.Nt"], p["dwf.Nx"], p["dwf.N5"], p["dwf.M5"], p["dwf.mf"])
    th, psi = g.npy("in_theta.npy"), g.field("in_psi.npy")
    rhs = d.apply_D_dagger(th, psi)
    r = d.conjugate_gradient(3, th, rhs, rtol=p["dwf.propagator_rtol"],
                             maxiter=p["dwf.propagator_maxiter"])
    info = g.npy("out_cg_info.npy")
    assert r.converged and abs(r.iterations - info[0]) <= 2
    assert rel(r.x, g.field("out_cg_x.npy")) < 1e-11
    assert r.info["true_relres"] < 1e-11


@pytest.mark.parametrize("op", [2, 3])
def test_cg64_matches_oracle_same_algorithm(tdwf, op):
    rng = np.random.default_rng(10 + op)
    Nt, Nx, Ls = 16, 16, 8
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.0, 0.1)
    o = O.Dwf(Nt, Nx, Ls, 1.0, 0.1)
    th = random_theta(rng, Nt, Nx)
    b = random_field(rng, o.ndof)
    xg = d.conjugate_gradient(op, th, b, rtol=1e-13, maxiter=5000)
    xo, it, rr, st = o.cg(op, th, b, 1e-13, 5000)
    assert st == 0 and xg.converged
    assert abs(xg.iterations - it) <= max(2, it // 50)
    assert rel(xg.x, xo) < 1e-12
    # stopping rule met on the recursive residual, true residual close to it
    assert xg.relative_residual <= 1e-13 and xg.info["true_relres"] < 1e-12


def test_cg_warm_start_and_edge_cases(tdwf):
    rng = np.random.default_rng(7)
    Nt, Nx, Ls = 8, 8, 4
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.0, 0.1)
    o = O.Dwf(Nt, Nx, Ls, 1.0, 0.1)
    th = random_theta(rng, Nt, Nx)
    b = random_field(rng, o.ndof)
    guess = random_field(rng, o.ndof) * 0.01
    xg = d.conjugate_gradient(2, th, b, initial_guess=guess, rtol=1e-12, maxiter=3000)
    xo, it, rr, st = o.cg(2, th, b, 1e-12, 3000, guess=guess)
    assert xg.converged and abs(xg.iterations - it) <= 2 and rel(xg.x, xo) < 1e-10
    # zero right-hand side: immediate return with x = guess (cg_solver.hpp:30-32)
    z = d.conjugate_gradient(3, th, np.zeros(o.ndof, complex), rtol=1e-10, maxiter=10)
    assert z.converged and z.iterations == 0 and not np.any(z.x)
    # maxiter reached: not converged, iterations == maxiter (cg_solver.hpp:63)
    m = d.conjugate_gradient(3, th, b, rtol=1e-14, maxiter=5)
    xo, it, rr, st = o.cg(3, th, b, 1e-14, 5)
    assert not m.converged and m.iterations == 5 and st == 1 and rel(m.x, xo) < 1e-12
    # guess already converged: zero iterations
    sol = d.conjugate_gradient(3, th, b, rtol=1e-12, maxiter=3000)
    again = d.conjugate_gradient(3, th, b, initial_guess=sol.x, rtol=1e-10, maxiter=3000)
    assert again.converged and again.iterations == 0


@pytest.mark.parametrize("shape", [(16, 16, 8), (32, 24, 12)])
def test_mixed_precision_reaches_fp64_true_residual(tdwf, shape):
    Nt, Nx, Ls = shape
    rng = np.random.default_rng(sum(shape))
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.0, 0.05)
    o = O.Dwf(Nt, Nx, Ls, 1.0, 0.05)
    th = random_theta(rng, Nt, Nx)
    b = random_field(rng, o.ndof)
    r = d.conjugate_gradient(3, th, b, rtol=1e-10, maxiter=20000, solver=tdwf.SOLVER_MIXED)
    assert r.converged and r.info["true_relres"] <= 1e-10
    assert r.info["reliable_updates"] >= 1
    ref = d.conjugate_gradient(3, th, b, rtol=1e-12, maxiter=20000)
    # both solutions within the conditioning of the solve
    assert rel(r.x, ref.x) < 1e-7


def test_batched_solve_many_configs(tdwf):
    """One persistent launch, right-hand sides on different configurations,
    each with its own convergence; every solution equals its own single
    solve on the oracle."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(21)
    Nt, Nx, Ls = 12, 8, 4
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.0, 0.1)
    o = O.Dwf(Nt, Nx, Ls, 1.0, 0.1)
    nconf, nrhs = 3, 7
    ths = np.stack([random_theta(rng, Nt, Nx) for _ in range(nconf)])
    d.set_gauge(ths)
    conf = np.array([k % nconf for k in range(nrhs)], np.int32)
    bs = np.stack([random_field(rng, o.ndof) * (k + 1) for k in range(nrhs)])
    b_t = torch.from_numpy(bs.view(np.float64).copy()).cuda()
    for solver in (tdwf.SOLVER_CG64, tdwf.SOLVER_MIXED):
        x_t = torch.zeros_like(b_t)
        infos = d.cg_batch_dev(3, b_t, x_t, rhs_conf=conf, rtol=1e-11, maxiter=4000,
                               solver=solver)
        xs = x_t.cpu().numpy().view(np.complex128).reshape(nrhs, -1)
        for k in range(nrhs):
            xo, it, rr, st = o.cg(3, ths[conf[k]], bs[k], 1e-12, 4000)
            assert infos[k]["converged"] and infos[k]["true_relres"] < 2e-11
            assert rel(xs[k], xo) < 1e-8
            if solver == tdwf.SOLVER_CG64:
                x1, it1, _, _ = o.cg(3, ths[conf[k]], bs[k], 1e-11, 4000)
                assert abs(infos[k]["iterations"] - it1) <= 2


def test_bounded_barrier_times_out_and_context_survives(tdwf):
    """A grid barrier that can never complete (more arrivals expected than
    blocks exist) ends in DWF_TIMEOUT after its limit; the same context then
    solves normally."""
    import time
    from three_part_dwf_study_b200 import _capi as A
    d = tdwf.DomainWall(8, 8, 4, 1.0, 0.1)
    assert A.lib().dwf_barrier_selftest(d.handle, 0, 1_000_000_000) == A.DWF_OK
    t0 = time.perf_counter()
    assert A.lib().dwf_barrier_selftest(d.handle, 1, 50_000_000) == A.DWF_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    assert "ran out" in A.lib().dwf_last_error(d.handle).decode()
    rng = np.random.default_rng(5)
    th = random_theta(rng, 8, 8)
    b = random_field(rng, d.Ndof)
    r = d.conjugate_gradient(3, th, b, rtol=1e-10, maxiter=2000)
    assert r.converged and r.info["true_relres"] < 1e-9


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("shape", [(8, 8, 4), (13, 37, 3), (64, 64, 16), (5, 3, 1), (16, 40, 24),
                                   (6, 32, 2), (3, 96, 5), (9, 128, 4), (20, 64, 1), (8, 32, 3),
                                   (16, 96, 1), (24, 64, 5)])
def test_dslash_variants_match_oracle(tdwf, variant, shape):
    """The Dslash kernels (one thread per 5-D site; one thread per 4-D site
    sweeping the fifth dimension; one thread per 5-D site with warp-shuffled x
    neighbours, which takes Nx % 32 == 0 and otherwise runs as the first; one
    thread per (s, x) sweeping a chunk of rows in t, which takes Nx % 32 == 0
    and Ls <= 16 and otherwise runs as the first; the Wilson-only row kernel,
    which runs as the first on domain wall; the column kernel with shuffled x
    neighbours, which takes Nx % 32 == 0 and otherwise runs as the second; the
    slice-ring kernel fed by bulk copies, which takes Nx % 32 == 0 and
    Nt % 8 == 0 and otherwise runs as the first: 8x32x3 is one block whose
    halo rows and columns all wrap) in FP64 and FP32, ragged
    tile edges, row/warp boundaries, several x tiles per block (9x128x4,
    20x64x1) and ragged t chunks included."""
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200 import _capi as A
    Nt, Nx, Ls = shape
    rng = np.random.default_rng(Nt * 7 + Nx * 3 + Ls)
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.2, 0.03)
    o = O.Dwf(Nt, Nx, Ls, 1.2, 0.03)
    assert A.lib().dwf_set_dslash_variant(d.handle, variant) == 0
    th = random_theta(rng, Nt, Nx)
    psi = random_field(rng, 2 * o.ndof)
    for op, name in OPS:
        ref = np.concatenate([o.apply(op, th, psi[:o.ndof]), o.apply(op, th, psi[o.ndof:])])
        assert rel(d.apply(op, th, psi), ref) < 1e-13, name
        x32 = torch.from_numpy(psi.astype(np.complex64)).cuda()
        y32 = torch.empty_like(x32)
        d.apply_dev(op, x32, y32)
        assert rel(y32.cpu().numpy(), ref) < 2e-6, name
    assert A.lib().dwf_dslash_variant(d.handle, 64, 2) == variant


@pytest.mark.parametrize("chunk", [1, 2, 3, 7, 13, 40])
@pytest.mark.parametrize("shape", [(13, 64, 6), (40, 32, 16)])
def test_dslash_sweep_chunks(tdwf, chunk, shape):
    """The t-sweeping Dslash at fixed chunk lengths: one-row chunks, chunks
    that do not divide Nt, and one chunk longer than Nt; three fields."""
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200 import _capi as A
    Nt, Nx, Ls = shape
    rng = np.random.default_rng(chunk * 31 + Nt)
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.7, 0.05)
    o = O.Dwf(Nt, Nx, Ls, 1.7, 0.05)
    assert A.lib().dwf_set_dslash_variant(d.handle, 3) == 0
    assert A.lib().dwf_set_dslash_chunk(d.handle, chunk) == 0
    th = random_theta(rng, Nt, Nx)
    psi = random_field(rng, 3 * o.ndof)
    for op, name in OPS:
        ref = np.concatenate([o.apply(op, th, psi[k * o.ndof:(k + 1) * o.ndof]) for k in range(3)])
        assert rel(d.apply(op, th, psi), ref) < 1e-13, name
        x32 = torch.from_numpy(psi.astype(np.complex64)).cuda()
        y32 = torch.empty_like(x32)
        d.apply_dev(op, x32, y32)
        assert rel(y32.cpu().numpy(), ref) < 2e-6, name
    assert A.lib().dwf_set_dslash_chunk(d.handle, -1) != 0


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("shape", [(16, 256), (7, 96), (12, 64), (4, 32), (8, 32), (36, 160)])
def test_wilson_dslash_variants_match_oracle(tdwf, variant, shape):
    """The Wilson operator (no fifth dimension, antiperiodic in both
    directions) through every Dslash kernel in FP64 and FP32; 16x256 puts
    eight 32-x tiles in one block of the t-sweeping kernel; for the row kernel
    (4 rows per thread, Nt % 4 == 0, else run as the site kernel) 4x32 is one
    warp whose halo rows and edge lanes both wrap, 7x96 the fallback, and
    36x160 leaves part of the last block without rows."""
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200 import _capi as A
    Nt, Nx = shape
    rng = np.random.default_rng(Nt + Nx)
    w = tdwf.Wilson(Nt, Nx, -0.3, 0.0, bc_t=-1.0, bc_x=-1.0)
    o = O.Wilson(Nt, Nx, -0.3, -1.0, -1.0)
    w.set_dslash_variant(variant)
    th = random_theta(rng, Nt, Nx)
    psi = random_field(rng, 2 * o.ntot)
    for op, name in OPS:
        ref = np.concatenate([o.apply(op, th, psi[:o.ntot]), o.apply(op, th, psi[o.ntot:])])
        assert rel(w.apply(op, th, psi), ref) < 1e-13, name
        x32 = torch.from_numpy(psi.astype(np.complex64)).cuda()
        y32 = torch.empty_like(x32)
        w.apply_dev(op, x32, y32)
        assert rel(y32.cpu().numpy(), ref) < 2e-6, name
    assert w.dslash_variant(32, 2) == variant
    with pytest.raises(A.DwfError):
        w.set_dslash_variant(7)


def test_wilson_dslash_autotuned_matches_oracle(tdwf):
    """The autotuner's pick on a 64x512 Wilson lattice (candidates include the
    t sweep at 16-, 32- and 64-row chunks with 16, 8 and 4 x tiles per block)
    agrees with the oracle in FP64 and FP32, one and three fields."""
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200 import _capi as A
    Nt, Nx = 64, 512
    rng = np.random.default_rng(64512)
    w = tdwf.Wilson(Nt, Nx, 0.05, 0.0)
    o = O.Wilson(Nt, Nx, 0.05, -1.0, 1.0)
    assert A.lib().dwf_set_dslash_variant(w.handle, -1) == 0
    th = random_theta(rng, Nt, Nx)
    for nf in (1, 3):
        psi = random_field(rng, nf * o.ntot)
        for op, name in OPS:
            ref = np.concatenate([o.apply(op, th, psi[k * o.ntot:(k + 1) * o.ntot])
                                  for k in range(nf)])
            assert rel(w.apply(op, th, psi), ref) < 1e-13, name
            x32 = torch.from_numpy(psi.astype(np.complex64)).cuda()
            y32 = torch.empty_like(x32)
            w.apply_dev(op, x32, y32)
            assert rel(y32.cpu().numpy(), ref) < 2e-6, name
        for prec in (64, 32):
            assert A.lib().dwf_dslash_variant(w.handle, prec, nf) in (0, 1, 2, 3, 4, 5)


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
def test_dslash_unaligned_fields(tdwf, variant):
    """FP64 fields that start 16 bytes past a 32-byte boundary (a view one
    complex number into a buffer) take the kernels' 16-byte access path; the
    results equal those of aligned fields."""
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200 import _capi as A
    Nt, Nx, Ls = (16 if variant == 6 else 12), 64, 4  # the slice ring takes Nt % 8 == 0
    rng = np.random.default_rng(77 + variant)
    d = tdwf.DomainWall(Nt, Nx, Ls, 1.3, 0.02)
    o = O.Dwf(Nt, Nx, Ls, 1.3, 0.02)
    assert A.lib().dwf_set_dslash_variant(d.handle, variant) == 0
    th = random_theta(rng, Nt, Nx)
    d.set_gauge(th)
    psi = random_field(rng, 2 * o.ndof)
    n = psi.size
    bx = torch.zeros(n + 1, dtype=torch.complex128, device="cuda")
    by = torch.zeros(n + 1, dtype=torch.complex128, device="cuda")
    x, y = bx[1:], by[1:]
    assert x.data_ptr() % 32 == 16 and y.data_ptr() % 32 == 16
    x.copy_(torch.from_numpy(psi))
    for op, name in OPS:
        ref = np.concatenate([o.apply(op, th, psi[:o.ndof]), o.apply(op, th, psi[o.ndof:])])
        d.apply_dev(op, x, y)
        assert rel(y.cpu().numpy(), ref) < 1e-13, name
        xa = torch.from_numpy(psi).cuda()
        ya = torch.empty_like(xa)
        d.apply_dev(op, xa, ya)
        assert rel(ya.cpu().numpy(), ref) < 1e-13, name


def test_apply_rejects_fields_off_16_byte_boundary(tdwf):
    """FP32 fields one complex number into a buffer (8 bytes past a 16-byte
    boundary) are refused with an error, not read by 16-byte accesses."""
    torch = pytest.importorskip("torch")
    from three_part_dwf_study_b200 import _capi as A
    w = tdwf.Wilson(8, 32, 0.1, 0.0)
    w.set_gauge(random_theta(np.random.default_rng(3), 8, 32))
    n = 8 * 32 * 2
    buf = torch.zeros(n + 1, dtype=torch.complex64, device="cuda")
    ok = torch.zeros(n, dtype=torch.complex64, device="cuda")
    assert buf[1:].data_ptr() % 16 == 8
    with pytest.raises(A.DwfError):
        w.apply_dev(0, buf[1:], ok)
    with pytest.raises(A.DwfError):
        w.apply_dev(0, ok, buf[1:])
    w.apply_dev(0, buf[:n], ok)
