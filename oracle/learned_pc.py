"""CPU restatement (float64 numpy) of the learned force-solve preconditioner.

TEST INFRASTRUCTURE ONLY: imported by tests/ to check the CUDA network's
loss and hand-written gradients (ibpm_b200/csrc/lpc.cu).  The reference has
no counterpart: it solves the moving-body force system with plain CG
(src/ConjugateGradientSolver.cc:35-65); the network only preconditions that
same solve, so what the oracle pins is the network arithmetic itself.

Network, per ordered pair (i, j) of boundary points:
  x_ij = [g_i, gbar_i, g_j, gbar_j, x_i - x_j, y_i - y_j, |p_i - p_j|]   19
  h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), k_ij = W3 h2 + b3         -> 4
g = (x, y, nx, ny) per point, gbar its mean over up to 8 boundary neighbours
(i +- 1..4, wrapping on closed curves).  Kraw[a P + i][c P + j] = k_ij[2a + c],
K = (Kraw + Kraw^T) / 2.  Loss: mean over configurations of
|K Mn - I|_F^2 / m with Mn = Mb / c0 (Mb = M / beta, c0 the last parameter).
"""
from __future__ import annotations

import numpy as np

K_F, K_H, K_O = 19, 256, 4
O_W1 = 0
O_B1 = O_W1 + K_H * K_F
O_W2 = O_B1 + K_H
O_B2 = O_W2 + K_H * K_H
O_W3 = O_B2 + K_H
O_B3 = O_W3 + K_O * K_H
O_C0 = O_B3 + K_O
N_PARAMS = O_C0 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[O_W1:O_B1].reshape(K_H, K_F), p[O_B1:O_W2], p[O_W2:O_B2].reshape(K_H, K_H), p[O_B2:O_W3],
            p[O_W3:O_B3].reshape(K_O, K_H), p[O_B3:O_C0], float(p[O_C0]))


def neighbours(bodies_xy):
    """Neighbour lists (nbr [P, 8], -1 padded; cnt [P]) for bodies given as
    [n, 2] point arrays; a body is closed when its end points are less than
    1.5 median spacings apart."""
    nbr, cnt, p0 = [], [], 0
    for xy in bodies_xy:
        xy = np.asarray(xy, dtype=np.float64).reshape(-1, 2)
        n = len(xy)
        d = np.sort(np.hypot(*(xy[1:] - xy[:-1]).T)) if n > 1 else np.zeros(0)
        med = d[len(d) // 2] if len(d) else 0.0
        gap = np.hypot(*(xy[-1] - xy[0])) if n > 1 else 0.0
        closed = n > 2 and gap < 1.5 * med
        for q in range(n):
            row = []
            for off in range(1, 5):
                for sgn in (-1, 1):
                    j = q + sgn * off
                    if closed:
                        j %= n
                    elif j < 0 or j >= n:
                        continue
                    if j == q:
                        continue
                    row.append(p0 + j)
            cnt.append(len(row))
            nbr.append(row + [-1] * (8 - len(row)))
        p0 += n
    return np.array(nbr, dtype=np.int64), np.array(cnt, dtype=np.int64)


def nbr_mean(g, nbr, cnt):
    """g [B, P, C] -> mean over each point's neighbours."""
    out = np.zeros_like(g)
    for q in range(8):
        has = cnt > q
        idx = np.where(has, nbr[:, q], 0)
        out += g[:, idx, :] * has[None, :, None]
    return out / np.maximum(cnt, 1)[None, :, None] * (cnt > 0)[None, :, None]


def pair_inputs(geom, nbr, cnt):
    g = np.asarray(geom, dtype=np.float64)
    B, P = g.shape[0], g.shape[1]
    gb = nbr_mean(g, nbr, cnt)
    gi = np.broadcast_to(g[:, :, None, :], (B, P, P, 4))
    gj = np.broadcast_to(g[:, None, :, :], (B, P, P, 4))
    bi = np.broadcast_to(gb[:, :, None, :], (B, P, P, 4))
    bj = np.broadcast_to(gb[:, None, :, :], (B, P, P, 4))
    d = gi[..., :2] - gj[..., :2]
    return np.concatenate([gi, bi, gj, bj, d, np.sqrt((d * d).sum(-1, keepdims=True))], axis=-1)  # [B,P,P,19]


def forward(params, geom, nbr, cnt):
    """K [B, m, m] (before the 1 / (c0 beta) scale) and the intermediates."""
    W1, b1, W2, b2, W3, b3, c0 = unpack(params)
    X = pair_inputs(geom, nbr, cnt)
    B, P = X.shape[0], X.shape[1]
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    k = h2 @ W3.T + b3                                              # [B,P,P,4]
    Kraw = k.reshape(B, P, P, 2, 2).transpose(0, 3, 1, 4, 2).reshape(B, 2 * P, 2 * P)
    K = 0.5 * (Kraw + Kraw.transpose(0, 2, 1))
    return K, dict(X=X, h1=h1, h2=h2, c0=c0)


def loss_grad(params, geom, mb, nbr, cnt):
    """Mean loss and its gradient with respect to the packed parameters (the c0 entry gets 0)."""
    W1, b1, W2, b2, W3, b3, c0 = unpack(params)
    K, c = forward(params, geom, nbr, cnt)
    B, m = K.shape[0], K.shape[1]
    P = m // 2
    Mn = np.asarray(mb, dtype=np.float64) / c0
    E = K @ Mn - np.eye(m)
    loss = float(np.mean(np.sum(E * E, axis=(1, 2)) / m))
    dE = 2.0 * E / (B * m)
    dK = dE @ Mn.transpose(0, 2, 1)
    dKraw = 0.5 * (dK + dK.transpose(0, 2, 1))
    dk = dKraw.reshape(B, 2, P, 2, P).transpose(0, 2, 4, 1, 3).reshape(B, P, P, 4)
    X, h1, h2 = c["X"], c["h1"], c["h2"]
    g = np.zeros(N_PARAMS)
    g[O_W3:O_B3] = np.einsum("bijq,bijk->qk", dk, h2).ravel()
    g[O_B3:O_C0] = dk.sum(axis=(0, 1, 2))
    dh2 = (dk @ W3) * (h2 > 0)
    g[O_W2:O_B2] = np.einsum("bijo,bijk->ok", dh2, h1).ravel()
    g[O_B2:O_W3] = dh2.sum(axis=(0, 1, 2))
    dh1 = (dh2 @ W2) * (h1 > 0)
    g[O_W1:O_B1] = np.einsum("bijo,bijk->ok", dh1, X).ravel()
    g[O_B1:O_W2] = dh1.sum(axis=(0, 1, 2))
    return loss, g


def operator(params, geom, nbr, cnt, beta):
    """The preconditioner matrix K / (c0 beta) for one configuration geom [P, 4]."""
    K, c = forward(params, np.asarray(geom)[None], nbr, cnt)
    return K[0] / (c["c0"] * beta)
