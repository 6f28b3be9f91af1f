"""CPU checks of the learned-preconditioner oracle itself: the gradient
against central finite differences, the adjoint chain against the inner
product identity, gauge covariance of the transports, and the BF16 rounding
rule. These pin the oracle that the GPU kernels are then compared with."""
import numpy as np
import pytest

from oracle import learned as LN


def rand_c(rng, *shape):
    return rng.normal(size=shape) + 1j * rng.normal(size=shape)


def small_net(rng, C0=4, H=3):
    ch = [C0, H, H, H, C0]
    return [0.3 * rand_c(rng, 9, ch[l + 1], ch[l]) for l in range(4)]


@pytest.fixture
def lat():
    rng = np.random.default_rng(5)
    Nt, Nx = 4, 6
    th = rng.uniform(-np.pi, np.pi, 2 * Nt * Nx)
    return Nt, Nx, th, LN.transports(th, Nt, Nx, -1.0, 1.0), LN.neighbours(Nt, Nx)


def test_bf16_rounding_ties_to_even():
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)  # bf16 spacing at 1
    vals = np.array([one + ulp / 2, one + 3 * ulp / 2, one + ulp / 4, -(one + 3 * ulp / 2)],
                    np.float32)
    np.testing.assert_array_equal(LN.bf16(vals),
                                  np.array([1.0, 1.0 + 2 * ulp, 1.0, -(1.0 + 2 * ulp)], np.float32))


def test_layout_round_trip():
    rng = np.random.default_rng(1)
    V, C = 12, 6
    f = rand_c(rng, 2, C // 2 * V * 2)
    np.testing.assert_array_equal(LN.from_net(LN.to_net(f, V, C), V, C), f)
    # channel c = 2*s + spin of site h sits at (s*V + h)*2 + spin
    g = LN.to_net(f, V, C)
    assert g[1, 5, 2 * 2 + 1] == f[1, (2 * V + 5) * 2 + 1]


def test_adjoint_identity(lat):
    Nt, Nx, th, T, nb = lat
    rng = np.random.default_rng(2)
    Ws = small_net(rng)
    V = Nt * Nx
    f = rand_c(rng, 2, V, 4)
    g = rand_c(rng, 2, V, 4)
    Nf, _ = LN.forward(T, nb, Ws, f, rounded=False)
    Ntg = LN.adjoint(T, nb, Ws, g, rounded=False)
    assert abs(np.vdot(g, Nf) - np.vdot(Ntg, f)) < 1e-10 * abs(np.vdot(g, Nf))


def test_gauge_covariance(lat):
    Nt, Nx, th, T, nb = lat
    rng = np.random.default_rng(3)
    Ws = small_net(rng)
    V = Nt * Nx
    phi = rng.uniform(-np.pi, np.pi, (Nt, Nx))
    t3 = th.reshape(2, Nt, Nx)
    th2 = np.stack([t3[0] + phi - np.roll(phi, -1, 0), t3[1] + phi - np.roll(phi, -1, 1)])
    T2 = LN.transports(th2.ravel(), Nt, Nx, -1.0, 1.0)
    f = rand_c(rng, 1, V, 4)
    ph = np.exp(1j * phi.ravel())[None, :, None]
    out1, _ = LN.forward(T, nb, Ws, f, rounded=False)
    out2, _ = LN.forward(T2, nb, Ws, ph * f, rounded=False)
    assert np.max(np.abs(out2 - ph * out1)) < 1e-12 * np.max(np.abs(out1))


def test_transport_reverse_is_conjugate(lat):
    Nt, Nx, th, T, nb = lat
    for k in range(9):
        np.testing.assert_allclose(T[:, LN.REV[k]], np.conj(T[nb[:, LN.REV[k]], k]), atol=1e-15)


def test_gradient_against_finite_differences(lat):
    Nt, Nx, th, T, nb = lat
    rng = np.random.default_rng(4)
    Ws = small_net(rng)
    V = Nt * Nx
    rho = rand_c(rng, 3, V, 4)
    e = rand_c(rng, 3, V, 4)
    _, grads = LN.loss_grad(T, nb, Ws, rho, e, rounded=False)
    h = 1e-6
    for li in range(4):
        for idx in [(0, 0, 0), (4, 1, 2), (8, 2, 1), (5, 0, 2)]:
            idx = tuple(min(i, s - 1) for i, s in zip(idx, Ws[li].shape))
            for unit, part in ((1.0, "re"), (1j, "im")):
                Wp = [w.copy() for w in Ws]
                Wm = [w.copy() for w in Ws]
                Wp[li][idx] += unit * h
                Wm[li][idx] -= unit * h
                lp, _ = LN.loss_grad(T, nb, Wp, rho, e, rounded=False)
                lm, _ = LN.loss_grad(T, nb, Wm, rho, e, rounded=False)
                fd = (lp - lm) / (2 * h)
                an = grads[li][idx].real if part == "re" else grads[li][idx].imag
                assert abs(fd - an) < 1e-6 * max(1.0, abs(an)), (li, idx, part, fd, an)


def test_rounded_mode_close_to_exact(lat):
    Nt, Nx, th, T, nb = lat
    rng = np.random.default_rng(6)
    Ws = small_net(rng)
    f = rand_c(rng, 2, Nt * Nx, 4)
    a, _ = LN.forward(T, nb, Ws, f, rounded=True)
    b, _ = LN.forward(T, nb, Ws, f, rounded=False)
    err = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert 1e-5 < err < 2e-2  # BF16 operands: about 2^-8 relative per layer
