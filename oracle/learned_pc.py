"""CPU restatement (float64 numpy) of the learned force-solve preconditioner.

TEST INFRASTRUCTURE ONLY: imported by tests/ to check the CUDA network's
loss and hand-written gradients (ibpm_b200/csrc/lpc.cu).  The reference has
no counterpart: it solves the moving-body force system with plain CG
(src/ConjugateGradientSolver.cc:35-65); the network only preconditions that
same solve, so what the oracle pins is the network arithmetic itself.

Network (per boundary point i, N(i) = up to 8 neighbours i +- 1..4 along the
body, wrapping on closed curves):
  a_i  = (x, y, nx, ny, rx/s, ry/s),  s = rms(r)
  h1_i = relu(W1 [a_i | mean_N a_j] + b1)          12 -> 256
  h2_i = relu(W2 [h1_i | mean_N h1_j] + b2)        512 -> 256
  o_i  = W3 h2_i + b3                               256 -> 2
Loss: mean over samples of |o - t|^2 / (|t|^2 + 1e-12), t = zb / s.
"""
from __future__ import annotations

import numpy as np

K_IN, K_IN2, K_H, K_H2, K_OUT = 6, 12, 256, 512, 2
O_W1 = 0
O_B1 = O_W1 + K_H * K_IN2
O_W2 = O_B1 + K_H
O_B2 = O_W2 + K_H * K_H2
O_W3 = O_B2 + K_H
O_B3 = O_W3 + K_OUT * K_H
N_PARAMS = O_B3 + K_OUT


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[O_W1:O_B1].reshape(K_H, K_IN2), p[O_B1:O_W2], p[O_W2:O_B2].reshape(K_H, K_H2), p[O_B2:O_W3],
            p[O_W3:O_B3].reshape(K_OUT, K_H), p[O_B3:N_PARAMS])


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


def _nbr_mean(x, nbr, cnt):
    """x [B, P, C] -> mean over each point's neighbours."""
    out = np.zeros_like(x)
    for q in range(8):
        has = cnt > q
        idx = np.where(has, nbr[:, q], 0)
        out += x[:, idx, :] * has[None, :, None]
    return out / np.maximum(cnt, 1)[None, :, None] * (cnt > 0)[None, :, None]


def forward(params, geom, r, nbr, cnt):
    """Outputs o [B, P, 2] and the intermediates of one batch."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    geom = np.asarray(geom, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    B, P = r.shape[0], r.shape[1] // 2
    s = np.sqrt(np.mean(r * r, axis=1)) + 1e-30
    feats = np.concatenate([geom, (r[:, :P] / s[:, None])[..., None], (r[:, P:] / s[:, None])[..., None]], axis=2)
    A = np.concatenate([feats, _nbr_mean(feats, nbr, cnt)], axis=2)        # [B, P, 12]
    h1 = np.maximum(A @ W1.T + b1, 0.0)
    C = np.concatenate([h1, _nbr_mean(h1, nbr, cnt)], axis=2)               # [B, P, 512]
    h2 = np.maximum(C @ W2.T + b2, 0.0)
    o = h2 @ W3.T + b3
    return o, dict(s=s, A=A, h1=h1, C=C, h2=h2)


def loss_grad(params, geom, r, zb, nbr, cnt):
    """Mean loss and its gradient with respect to the packed parameters."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    o, c = forward(params, geom, r, nbr, cnt)
    B, P = o.shape[0], o.shape[1]
    zb = np.asarray(zb, dtype=np.float64)
    t = np.stack([zb[:, :P], zb[:, P:]], axis=2) / c["s"][:, None, None]   # [B, P, 2]
    e = o - t
    denom = np.sum(t * t, axis=(1, 2)) + 1e-12
    loss = np.mean(np.sum(e * e, axis=(1, 2)) / denom)
    do = 2.0 * e / (denom[:, None, None] * B)
    g = np.zeros(N_PARAMS)
    h2, C, h1, A = c["h2"], c["C"], c["h1"], c["A"]
    g[O_W3:O_B3] = np.einsum("bpc,bpk->ck", do, h2).ravel()
    g[O_B3:N_PARAMS] = do.sum(axis=(0, 1))
    dh2 = (do @ W3) * (h2 > 0)
    g[O_W2:O_B2] = np.einsum("bpo,bpk->ok", dh2, C).ravel()
    g[O_B2:O_W3] = dh2.sum(axis=(0, 1))
    dC = dh2 @ W2
    # the neighbour mean's adjoint: point j receives dC_i[256:] / cnt_i from every i with j in N(i)
    dmean = dC[:, :, K_H:] / np.maximum(cnt, 1)[None, :, None]
    dh1 = dC[:, :, :K_H].copy()
    for q in range(8):
        has = cnt > q
        for i in np.nonzero(has)[0]:
            dh1[:, nbr[i, q], :] += dmean[:, i, :]
    dh1 *= h1 > 0
    g[O_W1:O_B1] = np.einsum("bpo,bpk->ok", dh1, A).ravel()
    g[O_B1:O_W2] = dh1.sum(axis=(0, 1))
    return loss, g


def apply(params, geom, r, nbr, cnt, beta):
    """z = (s / beta) o for one residual r [2P] (the preconditioner action)."""
    o, c = forward(params, geom[None], np.asarray(r, dtype=np.float64)[None], nbr, cnt)
    return np.concatenate([o[0, :, 0], o[0, :, 1]]) * c["s"][0] / beta
