"""CPU restatement of the learned preconditioner network (TEST INFRASTRUCTURE ONLY).

The network has no counterpart in the reference; this module defines its
arithmetic in numpy so that the GPU kernels can be checked against it:

* a parallel-transport convolution (PTC) layer maps a field with Cin complex
  channels per lattice site to one with Cout channels,
      out(y)[o] = sum_k sum_i W_k[o][i] * a_k(y)[i],
      a_k(y)[i] = T_k(y) * in(y + d_k)[i],
  over the nine offsets d_k of a 3x3 stencil, where T_k(y) is the U(1)
  parallel transporter from y + d_k to y (fermion boundary signs included;
  the diagonal offsets average the two two-link paths);
* the network is four such layers, C0 -> H -> H -> H -> C0, without bias or
  activation, so it is linear and gauge covariant, and its adjoint is the
  same chain run backwards with W'_k = (W_rev(k))^H;
* the GPU evaluates a layer as out(y) = sum_k T_k(y) P_k(y + d_k) with
  P_k = W_k in: the input field and the weights are rounded to BF16 (round to
  nearest even), P_k is accumulated in FP32 on the tensor cores, and the
  transporter products and the sum over k are FP32; ``rounded=True``
  reproduces the rounding of the operands exactly and accumulates in FP64,
  ``rounded=False`` is the exact FP64 network used for the finite-difference
  gradient checks.

Fields enter and leave in the operator's own layout (domain wall: index
((s*Nt+t)*Nx+x)*2+spin, channel c = 2*s+spin; Wilson: (t*Nx+x)*2+spin,
channel c = spin); hidden fields are [V][H].
"""
import numpy as np

OFFSETS = ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (1, -1), (-1, 1), (-1, -1))
REV = (0, 2, 1, 4, 3, 8, 7, 6, 5)


def neighbours(Nt, Nx):
    """nb[h, k]: site index of (t + dt_k, x + dx_k), periodic."""
    t = np.arange(Nt)[:, None] + np.zeros((1, Nx), int)
    x = np.arange(Nx)[None, :] + np.zeros((Nt, 1), int)
    nb = np.zeros((Nt * Nx, 9), np.int64)
    for k, (dt, dx) in enumerate(OFFSETS):
        nb[:, k] = (((t + dt) % Nt) * Nx + (x + dx) % Nx).ravel()
    return nb


def transports(theta, Nt, Nx, bct, bcx):
    """T[h, k] (complex128): transporter from site h + d_k to h."""
    th = np.asarray(theta, np.float64).reshape(2, Nt, Nx)
    U = np.cos(th) + 1j * np.sin(th)
    t = np.arange(Nt)[:, None] + np.zeros((1, Nx), int)
    x = np.arange(Nx)[None, :] + np.zeros((Nt, 1), int)

    def hop(mu, sg, tt, xx):
        # one hop from (tt, xx) along +-mu, as seen from (tt, xx)
        if mu == 0:
            if sg > 0:
                return U[0, tt % Nt, xx % Nx] * np.where(tt % Nt == Nt - 1, bct, 1.0)
            return np.conj(U[0, (tt - 1) % Nt, xx % Nx]) * np.where(tt % Nt == 0, bct, 1.0)
        if sg > 0:
            return U[1, tt % Nt, xx % Nx] * np.where(xx % Nx == Nx - 1, bcx, 1.0)
        return np.conj(U[1, tt % Nt, (xx - 1) % Nx]) * np.where(xx % Nx == 0, bcx, 1.0)

    T = np.zeros((Nt, Nx, 9), np.complex128)
    for k, (dt, dx) in enumerate(OFFSETS):
        if dt == 0 and dx == 0:
            T[:, :, k] = 1.0
        elif dx == 0:
            T[:, :, k] = hop(0, dt, t, x)
        elif dt == 0:
            T[:, :, k] = hop(1, dx, t, x)
        else:
            p1 = hop(0, dt, t, x) * hop(1, dx, t + dt, x)
            p2 = hop(1, dx, t, x) * hop(0, dt, t, x + dx)
            T[:, :, k] = 0.5 * (p1 + p2)
    return T.reshape(Nt * Nx, 9)


def bf16(a):
    """Round float32 values to the nearest bfloat16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16c(z):
    """Round both parts of a complex array to bfloat16 (complex128 result)."""
    z = np.asarray(z)
    return bf16(z.real.astype(np.float32)).astype(np.float64) + \
        1j * bf16(z.imag.astype(np.float32)).astype(np.float64)


def to_net(f, V, C):
    """Operator layout (flat, per right-hand side) -> [B, V, C]."""
    f = np.asarray(f).reshape(-1, C // 2, V, 2)
    return np.ascontiguousarray(f.transpose(0, 2, 1, 3).reshape(-1, V, C))


def from_net(g, V, C):
    """[B, V, C] -> operator layout [B, C//2 * V * 2]."""
    g = np.asarray(g).reshape(-1, V, C // 2, 2)
    return np.ascontiguousarray(g.transpose(0, 2, 1, 3).reshape(g.shape[0], -1))


def gather(T, nb, fin, k, rounded):
    """a_k = T_k * fin(neighbour k) for fin [B, V, Cin] (fin rounded to BF16
    when rounded)."""
    v = fin[:, nb[:, k], :]
    t = T[:, k][None, :, None]
    if rounded:
        return t * bf16c(v)
    return t * v


def layer(T, nb, W, fin, rounded=True):
    """One PTC layer: W [9, Cout, Cin] complex, fin [B, V, Cin] -> [B, V, Cout]."""
    Wr = bf16c(W) if rounded else W
    out = 0
    for k in range(9):
        out = out + np.einsum('oi,bvi->bvo', Wr[k], gather(T, nb, fin, k, rounded))
    return out


def adjoint_weights(W):
    """Weights of the adjoint layer: W'_k = (W_rev(k))^H, shape [9, Cin, Cout]."""
    return np.ascontiguousarray(np.conj(np.asarray(W)[list(REV)]).transpose(0, 2, 1))


def forward(T, nb, Ws, fin, rounded=True):
    """Network output and the input of each layer (inputs stored as the GPU
    stores them: complex64 when rounded)."""
    acts = []
    f = fin
    for W in Ws:
        f = f.astype(np.complex64) if rounded else f
        acts.append(f)
        f = layer(T, nb, W, f, rounded)
    return f, acts


def adjoint(T, nb, Ws, g, rounded=True):
    for W in reversed(Ws):
        g = g.astype(np.complex64) if rounded else g
        g = layer(T, nb, adjoint_weights(W), g, rounded)
    return g


def loss_grad(T, nb, Ws, rho, e, rounded=True):
    """Loss (1/B) sum_b |N rho_b - e_b|^2 / |e_b|^2 and its gradient with
    respect to each layer's weights, dL/dRe W + i dL/dIm W.

    rho, e: [B, V, C0]. In rounded mode the output and every back-propagated
    field are held in complex64 as on the GPU."""
    out, acts = forward(T, nb, Ws, rho, rounded)
    B = rho.shape[0]
    ee = np.sum(np.abs(e) ** 2, axis=(1, 2))
    diff = (out.astype(np.complex64) if rounded else out) - e
    loss = float(np.sum(np.sum(np.abs(diff) ** 2, axis=(1, 2)) / ee) / B)
    g = 2.0 * diff / (B * ee)[:, None, None]
    grads = [None] * len(Ws)
    for li in range(len(Ws) - 1, -1, -1):
        g = g.astype(np.complex64) if rounded else g
        fin = acts[li]
        G = np.zeros_like(Ws[li], dtype=np.complex128)
        for k in range(9):
            a = gather(T, nb, fin, k, rounded)
            G[k] = np.einsum('bvo,bvi->oi', g, np.conj(a))
        grads[li] = G
        g = layer(T, nb, adjoint_weights(Ws[li]), g, rounded)
    return loss, grads
