"""Learned preconditioner on the GPU: the network kernels against the CPU
oracle (transports, each layer and its adjoint, the whole network, loss and
weight gradients), training on the GPU, and the preconditioned solve: it
meets the reference's stopping rule, reproduces the FP64 solution, and the
trained network saves iterations over the untrained one (the ablation)."""
import numpy as np
import pytest

from conftest import quenched_theta, rel
from oracle import learned as LN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import three_part_dwf_study_b200 as T
    return T


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def setup_dwf(T, Nt=8, Nx=12, Ls=4, hidden=8, seed=3, nconf=2, beta=2.0):
    rng = np.random.default_rng(seed)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.1)
    th = np.stack([quenched_theta(rng, Nt, Nx, beta) for _ in range(nconf)])
    d.set_gauge(th)
    d.lp_init(hidden=hidden, seed=seed)
    # perturb the weights so every entry matters
    ws = [w + (0.05 * (rng.normal(size=w.shape) + 1j * rng.normal(size=w.shape))).astype(np.complex64)
          for w in d.lp_weights()]
    d.lp_set_weights(ws)
    return d, th, d.lp_weights()


def crand(rng, *shape):
    return (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)


def test_transports_match_oracle(T):
    d, th, _ = setup_dwf(T)
    for c in range(2):
        Tg = d.lp_transports(c)
        To = LN.transports(th[c], d.Nt, d.Nx, -1.0, 1.0)
        assert np.max(np.abs(Tg - To)) < 2e-7
    d.close()


@pytest.mark.parametrize("variant", [1, 0])
@pytest.mark.parametrize("adjoint", [False, True])
def test_each_layer_matches_oracle(T, torch, adjoint, variant):
    """Both layer kernels (1: tcgen05 with TMEM accumulators, 0: mma.sync)."""
    d, th, ws = setup_dwf(T)
    d.lp_set_variant(variant)
    rng = np.random.default_rng(11)
    V = d.Nt * d.Nx
    nb = LN.neighbours(d.Nt, d.Nx)
    conf = np.array([1, 0, 1], np.int32)
    for l, W in enumerate(ws):
        Wl = LN.adjoint_weights(W) if adjoint else W
        cin = Wl.shape[2]
        cout = Wl.shape[1]
        x = crand(rng, 3, V, cin)
        out = torch.empty((3, V, cout), dtype=torch.complex64, device="cuda")
        d.lp_layer_dev(l, torch.from_numpy(x).cuda(), out, adjoint=adjoint, rhs_conf=conf)
        got = out.cpu().numpy()
        for b in range(3):
            Tg = d.lp_transports(int(conf[b])).astype(np.complex128)
            ref = LN.layer(Tg, nb, W if not adjoint else Wl, x[b:b + 1], rounded=True)[0]
            # same BF16 operands; FP32 vs FP64 accumulation only
            assert rel(got[b], ref) < 2e-6, (l, b)
    d.close()


@pytest.mark.parametrize("variant", [1, 0])
def test_network_matches_oracle(T, torch, variant):
    d, th, ws = setup_dwf(T)
    d.lp_set_variant(variant)
    rng = np.random.default_rng(12)
    V, C0 = d.Nt * d.Nx, 2 * d.Ls
    nb = LN.neighbours(d.Nt, d.Nx)
    f = crand(rng, 2, d.Ndof)
    out = torch.empty((2, d.Ndof), dtype=torch.complex64, device="cuda")
    Tg = d.lp_transports(0).astype(np.complex128)
    for adjoint in (False, True):
        d.lp_apply_dev(torch.from_numpy(f).cuda(), out, adjoint=adjoint)
        got = out.cpu().numpy()
        fin = LN.to_net(f, V, C0)
        if adjoint:
            ref = LN.adjoint(Tg, nb, ws, fin, rounded=True)
            exact = LN.adjoint(Tg, nb, ws, fin, rounded=False)
        else:
            ref = LN.forward(Tg, nb, ws, fin, rounded=True)[0]
            exact = LN.forward(Tg, nb, ws, fin, rounded=False)[0]
        ref = LN.from_net(ref, V, C0)
        exact = LN.from_net(exact, V, C0)
        # identical rounding chain: only rare BF16 ties differ after FP32 accumulation
        assert rel(got, ref) < 1e-3
        # BF16 operands against the exact FP64 network: about 2^-8 per layer
        assert rel(got, exact) < 3e-2
    d.close()


@pytest.mark.parametrize("variant", [1, 0])
def test_loss_and_gradient_match_oracle(T, torch, variant):
    d, th, ws = setup_dwf(T)
    d.lp_set_variant(variant)
    rng = np.random.default_rng(13)
    V, C0 = d.Nt * d.Nx, 2 * d.Ls
    nb = LN.neighbours(d.Nt, d.Nx)
    rho = crand(rng, 3, d.Ndof)
    e = crand(rng, 3, d.Ndof)
    conf = np.array([0, 0, 0], np.int32)
    loss, grads = d.lp_loss_grad_dev(torch.from_numpy(rho).cuda(), torch.from_numpy(e).cuda(),
                                     pair_conf=conf)
    Tg = d.lp_transports(0).astype(np.complex128)
    lo, go = LN.loss_grad(Tg, nb, ws, LN.to_net(rho, V, C0), LN.to_net(e, V, C0), rounded=True)
    assert abs(loss - lo) < 1e-5 * abs(lo)
    for l in range(4):
        assert rel(grads[l], go[l]) < 2e-3, l
    # and the oracle's rounded gradient is close to the exact one
    _, gx = LN.loss_grad(Tg, nb, ws, LN.to_net(rho, V, C0), LN.to_net(e, V, C0), rounded=False)
    for l in range(4):
        assert rel(grads[l], gx[l]) < 5e-2, l
    d.close()


def test_gradient_matches_oracle_at_the_widest_layers(T, torch):
    """Ls = 24 with 32 hidden channels (48 x 32 complex weights per offset,
    the weight-gradient kernel's wider per-thread tiling): loss and gradient
    against the oracle's rounded network."""
    d, th, ws = setup_dwf(T, Nt=8, Nx=12, Ls=24, hidden=32)
    rng = np.random.default_rng(31)
    V, C0 = d.Nt * d.Nx, 2 * d.Ls
    nb = LN.neighbours(d.Nt, d.Nx)
    rho = crand(rng, 2, d.Ndof)
    e = crand(rng, 2, d.Ndof)
    conf = np.array([0, 1], np.int32)
    loss, grads = d.lp_loss_grad_dev(torch.from_numpy(rho).cuda(), torch.from_numpy(e).cuda(),
                                     pair_conf=conf)
    lo = 0.0
    go = [np.zeros_like(w, dtype=np.complex128) for w in ws]
    for b in range(2):
        Tg = d.lp_transports(int(conf[b])).astype(np.complex128)
        lb, gb = LN.loss_grad(Tg, nb, ws, LN.to_net(rho[b:b + 1], V, C0), LN.to_net(e[b:b + 1], V, C0),
                              rounded=True)
        lo += lb / 2
        for l in range(4):
            go[l] += gb[l] / 2
    assert abs(loss - lo) < 1e-5 * abs(lo)
    for l in range(4):
        assert rel(grads[l], go[l]) < 2e-3, l
    d.close()


@pytest.mark.parametrize("Ls,hidden,Nt,Nx", [(16, 32, 16, 64), (12, 24, 16, 64), (24, 16, 16, 64),
                                          (20, 24, 16, 64), (16, 32, 4, 256)])
def test_layer_variants_agree_at_wide_layers(T, torch, Ls, hidden, Nt, Nx):
    """tcgen05 and mma.sync networks on wide domain-wall fields agree to FP32
    accumulation order: the benchmark's widths (Ls = 16, hidden 32: 64 real
    columns, two CTAs per SM), 24 channels (48 columns, 8-column TMEM loads),
    48 channels (96 columns, one double-buffered CTA), 40 channels, and 32
    channels at Nx = 256 (one CTA per SM with a single window buffer: two
    buffers would exceed the shared memory)."""
    rng = np.random.default_rng(17 + Ls + hidden + Nx)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, 0.05)
    d.set_gauge(quenched_theta(rng, Nt, Nx, 3.0)[None])
    d.lp_init(hidden=hidden, seed=2)
    f = torch.from_numpy(crand(rng, 3, d.Ndof)).cuda()
    outs = []
    for v in (1, 0):
        d.lp_set_variant(v)
        o = torch.empty_like(f)
        d.lp_apply_dev(f, o)
        outs.append(o.cpu().numpy())
    assert rel(outs[0], outs[1]) < 1e-3
    d.close()


def test_training_reduces_loss(T):
    d, th, _ = setup_dwf(T, Nt=16, Nx=16, Ls=4, hidden=8)
    d.lp_init(hidden=8, seed=5)
    info, hist = d.lp_train(steps=300, batch=4, lr=3e-3, pairs_per_conf=16, solver_iters=20,
                            solver_every=2, seed=9, history=True)
    assert info["npairs"] == 32 and info["solver_pairs"] > 0
    assert np.all(np.isfinite(hist))
    assert np.mean(hist[-30:]) < 0.5 * np.mean(hist[:10])
    d.close()


def learned_setup(T, Nt, Nx, Ls, beta, hidden, steps, seed=21, mf=0.05):
    rng = np.random.default_rng(seed)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, mf)
    th = np.stack([quenched_theta(rng, Nt, Nx, beta) for _ in range(4)])
    d.set_gauge(th)
    d.lp_init(hidden=hidden, seed=seed)
    untrained = d.lp_weights()
    info = d.lp_train(steps=steps, batch=8, lr=3e-3, lr_decay_steps=steps // 2,
                      pairs_per_conf=32, solver_iters=30, solver_every=2, seed=seed)
    return d, th, untrained, info


def point_sources(Nt, Nx, Ls, n):
    src = np.zeros((n, Ls, Nt, Nx, 2), np.complex128)
    for k in range(n):
        src[k, 0, (4 * k) % Nt, 0, k % 2] = 1.0
        src[k, Ls - 1, (4 * k) % Nt, 0, k % 2] = 1.0
    return src.reshape(n, -1)


def test_learned_solve_meets_rule_and_matches_fp64(T):
    """More right-hand sides (10) than the training batch (8): the solver's
    buffers are sized for its own batch."""
    d, th, untrained, tinfo = learned_setup(T, 16, 16, 8, 3.0, 16, 600)
    src = point_sources(16, 16, 8, 10)
    conf = np.arange(10, dtype=np.int32) % 4
    x, info = d.propagators(src, rhs_conf=conf, rtol=1e-10, maxiter=20000, solver=T.SOLVER_LEARNED)
    x64, i64 = d.propagators(src, rhs_conf=conf, rtol=1e-12, maxiter=40000, solver=T.SOLVER_CG64)
    for k in range(10):
        assert info[k]["converged"] and info[k]["true_relres"] <= 1e-10, info[k]
        assert info[k]["solver"] == T.SOLVER_LEARNED and info[k]["fallback"] == 0
        assert rel(x[k], x64[k]) < 1e-7
    d.close()


def test_trained_network_beats_untrained_and_plain_cg(T):
    """Ablation: the same solver with the untrained (initial) weights needs
    more iterations; plain CG needs more operator applications."""
    d, th, untrained, tinfo = learned_setup(T, 16, 16, 8, 3.0, 16, 600)
    src = point_sources(16, 16, 8, 4)
    conf = np.array([0, 1, 2, 3], np.int32)
    _, tr = d.propagators(src, rhs_conf=conf, rtol=1e-10, maxiter=20000, solver=T.SOLVER_LEARNED)
    trained = d.lp_weights()
    d.lp_set_weights(untrained)
    _, un = d.propagators(src, rhs_conf=conf, rtol=1e-10, maxiter=20000, solver=T.SOLVER_LEARNED)
    d.lp_set_weights(trained)
    _, cg = d.propagators(src, rhs_conf=conf, rtol=1e-10, maxiter=40000, solver=T.SOLVER_CG64)
    it_tr = sum(i["schur_iterations"] for i in tr)
    it_un = sum(i["schur_iterations"] + (i["iterations"] - i["schur_iterations"]) for i in un)
    it_cg = sum(i["iterations"] for i in cg)
    assert all(i["converged"] for i in tr + un + cg)
    # D applications: learned 1 per GCR iteration, CG 2 per iteration
    assert it_tr < 0.7 * it_un
    assert it_tr < 0.5 * 2 * it_cg
    d.close()


@pytest.mark.parametrize("method,restart", [(0, 4), (0, 8), (0, 16), (1, 8)])
def test_learned_krylov_methods_meet_rule(T, method, restart):
    """Flexible GCR at each restart length and BiCGStab: every right-hand
    side meets the stopping rule on the FP64 true residual without the
    fallback and equals the FP64 solution."""
    d, th, untrained, tinfo = learned_setup(T, 16, 16, 8, 3.0, 16, 600)
    src = point_sources(16, 16, 8, 6)
    conf = np.arange(6, dtype=np.int32) % 4
    x64, _ = d.propagators(src, rhs_conf=conf, rtol=1e-12, maxiter=40000, solver=T.SOLVER_CG64)
    d.lp_set_krylov(method, restart)
    x, info = d.propagators(src, rhs_conf=conf, rtol=1e-10, maxiter=20000, solver=T.SOLVER_LEARNED)
    for k in range(6):
        assert info[k]["converged"] and info[k]["true_relres"] <= 1e-10, info[k]
        assert info[k]["fallback"] == 0 and info[k]["schur_iterations"] > 0
        assert rel(x[k], x64[k]) < 1e-7
    d.close()


def test_learned_krylov_rejects_bad_restart(T):
    d = T.DomainWall(8, 8, 4, 1.0, 0.1)
    d.set_gauge(np.zeros(2 * 64))
    d.lp_init(hidden=8, seed=1)
    for method, restart in ((0, 6), (0, 20), (0, 0), (2, 8)):
        with pytest.raises(T.DwfError):
            d.lp_set_krylov(method, restart)
    d.lp_set_krylov(1, 0)
    d.close()


def test_learned_wilson(T):
    rng = np.random.default_rng(4)
    w = T.Wilson(16, 16, 0.05, 2.0)
    th = np.stack([quenched_theta(rng, 16, 16, 3.0) for _ in range(2)])
    w.set_gauge(th)
    w.lp_init(hidden=8, seed=4)
    w.lp_train(steps=400, batch=8, lr=3e-3, lr_decay_steps=200, pairs_per_conf=32,
               solver_iters=20, seed=4)
    src = np.zeros((2, w.Ndof), np.complex128)
    src[0, 0] = 1.0
    src[1, 3] = 1.0
    x, info = w.propagators(src, rhs_conf=[0, 1], rtol=1e-10, maxiter=20000, solver=T.SOLVER_LEARNED)
    x64, i64 = w.propagators(src, rhs_conf=[0, 1], rtol=1e-12, maxiter=40000, solver=T.SOLVER_CG64)
    for k in range(2):
        assert info[k]["converged"] and info[k]["true_relres"] <= 1e-10
        assert rel(x[k], x64[k]) < 1e-7
        assert info[k]["schur_iterations"] < i64[k]["iterations"]
    w.close()


def test_learned_solve_kernel_choices_agree(T):
    """The learned solve with the mma.sync layer kernel, the tcgen05 layer
    kernel and the automatic choice (both timed at the first solve, the faster
    kept): every result meets the stopping rule and equals the FP64 solution."""
    rng = np.random.default_rng(9)
    w = T.Wilson(16, 32, -0.02, 3.0)
    th = np.stack([quenched_theta(rng, 16, 32, 3.0) for _ in range(2)])
    w.set_gauge(th)
    w.lp_init(hidden=8, seed=9)
    w.lp_train(steps=300, batch=8, lr=3e-3, lr_decay_steps=150, pairs_per_conf=32,
               solver_iters=20, seed=9)
    src = np.zeros((3, w.Ndof), np.complex128)
    for k in range(3):
        src[k, 2 * (5 * k * 32 + k) + (k % 2)] = 1.0
    conf = [0, 1, 0]
    x64, _ = w.propagators(src, rhs_conf=conf, rtol=1e-12, maxiter=40000, solver=T.SOLVER_CG64)
    for variant in (0, 1, -1, -1):
        w.lp_set_variant(variant)
        x, info = w.propagators(src, rhs_conf=conf, rtol=1e-10, maxiter=20000,
                                solver=T.SOLVER_LEARNED)
        for k in range(3):
            assert info[k]["converged"] and info[k]["true_relres"] <= 1e-10, (variant, info[k])
            assert rel(x[k], x64[k]) < 1e-7, variant
    w.close()
