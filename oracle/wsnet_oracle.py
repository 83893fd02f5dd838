"""CPU restatement of the steady-state warm-start network (test
infrastructure only; the product runs quac_b200/csrc/warmnet.cu).

Float64 numpy forward pass, loss  mean_s ||F_s F_s^H - rho_s||_F^2  and the
backward pass of the same network, used to check the GPU training kernels'
gradients.  Parameter order and layouts follow the product: W1 [H x 32]
(inputs padded from 4 to 32), b1 [H], W2 [H x H], b2 [H], W3 [2 D r x H],
b3 [2 D r]; output row s holds F_s column-major as (re, im) pairs.
There is no reference counterpart (QuaC has no learned component).
"""
import numpy as np

IN_PAD = 32


def unpack(p, D, r, H):
    O = 2 * D * r
    sizes = [H * IN_PAD, H, H * H, H, O * H, O]
    parts, off = [], 0
    for n in sizes:
        parts.append(np.asarray(p[off:off + n], dtype=np.float64))
        off += n
    W1, b1, W2, b2, W3, b3 = parts
    return W1.reshape(H, IN_PAD), b1, W2.reshape(H, H), b2, W3.reshape(O, H), b3


def forward(p, X, D, r, H):
    W1, b1, W2, b2, W3, b3 = unpack(p, D, r, H)
    Xp = np.zeros((X.shape[0], IN_PAD))
    Xp[:, :X.shape[1]] = X
    H1 = np.tanh(Xp @ W1.T + b1)
    H2 = np.tanh(H1 @ W2.T + b2)
    O = H2 @ W3.T + b3
    return Xp, H1, H2, O


def factors(O, D, r):
    """(n, 2 D r) network output -> (n, D, r) complex factors."""
    z = O[:, 0::2] + 1j * O[:, 1::2]
    return np.transpose(z.reshape(O.shape[0], r, D), (0, 2, 1))


def loss_grad(p, X, rhos, D, r, H):
    W1, b1, W2, b2, W3, b3 = unpack(p, D, r, H)
    Xp, H1, H2, O = forward(p, X, D, r, H)
    n = X.shape[0]
    F = factors(O, D, r)
    E = F @ np.conj(np.transpose(F, (0, 2, 1))) - rhos
    loss = float(np.sum(np.abs(E) ** 2)) / n
    dF = 4.0 * (E @ F) / n                       # real-pair gradient
    dO = np.zeros_like(O)
    dz = np.transpose(dF, (0, 2, 1)).reshape(n, D * r)
    dO[:, 0::2], dO[:, 1::2] = dz.real, dz.imag
    gW3, gb3 = dO.T @ H2, dO.sum(0)
    dZ2 = (dO @ W3) * (1 - H2 ** 2)
    gW2, gb2 = dZ2.T @ H1, dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * (1 - H1 ** 2)
    gW1, gb1 = dZ1.T @ Xp, dZ1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
