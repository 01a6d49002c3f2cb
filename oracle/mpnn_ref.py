"""CPU oracle of the learned preconditioner (message-passing network).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU
forward and backward kernels.  The product never imports it.

The reference has no learned part (it solves with Eigen::SparseLU,
corlib/SystemSolveEigenSparse.hpp:153); this module restates the network the
GPU library defines, in float64 numpy, with the operands of the three dense
layers rounded to BF16 at the same places the tensor-core kernels round them
(``bf16=True``), or unrounded (``bf16=False``, used for finite differences):

    Ahat = D^-1/2 S D^-1/2                    S: symmetric elimination operator
    x0   = D^-1/2 r / s,  s = rms(D^-1/2 r)
    H0   = relu(E [x0, Ahat x0] + e)
    Hl   = relu([H(l-1) | Ahat H(l-1)] Wl^T + bl),  l = 1..3
    yhat = x0 + H3 w + c  (x0 alone on constrained dofs)
    M(r) = s D^-1/2 yhat
    loss = d^T Ahat d / N,  d = yhat - D^1/2 e / s

Parameter layout (float32 vector): E [64][2], e [64], then per layer
W [64][128] (row = output feature) and b [64], then w [64], c.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

H = 64
LAYERS = 3
OFF_EW = 0
OFF_EB = OFF_EW + 2 * H
OFF_L = OFF_EB + H
LSZ = H * 2 * H + H
OFF_DW = OFF_L + LAYERS * LSZ
OFF_DB = OFF_DW + H
NPARAM = OFF_DB + 1


def bf16(a):
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def symmetric_operator(rp, col, val, mask):
    """S from the row-zeroed reference matrix: off-diagonal entries in a
    constrained row or column set to zero, diagonal kept."""
    N = len(rp) - 1
    A = sp.csr_matrix((np.asarray(val, dtype=np.float64), col, rp), shape=(N, N)).tocoo()
    m = np.asarray(mask, dtype=bool)
    keep = ~((m[A.row] | m[A.col]) & (A.row != A.col))
    v = np.where(keep, A.data, 0.0)
    return sp.csr_matrix((v, (A.row, A.col)), shape=(N, N))


def scaled_operator(S):
    """(Ahat, sdinv) with sdinv = float32(1/sqrt(diag S)) and Ahat values
    rounded to float32 like the device copy."""
    d = S.diagonal()
    si = 1.0 / np.sqrt(d)
    C = S.tocoo()
    v = (C.data * si[C.row] / np.sqrt(d[C.col])).astype(np.float32).astype(np.float64)
    Ahat = sp.csr_matrix((v, (C.row, C.col)), shape=S.shape)
    return Ahat, si.astype(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    E = p[OFF_EW:OFF_EW + 2 * H].reshape(H, 2)
    eb = p[OFF_EB:OFF_EB + H]
    W = [p[OFF_L + l * LSZ:OFF_L + l * LSZ + H * 2 * H].reshape(H, 2 * H) for l in range(LAYERS)]
    b = [p[OFF_L + l * LSZ + H * 2 * H:OFF_L + (l + 1) * LSZ] for l in range(LAYERS)]
    return E, eb, W, b, p[OFF_DW:OFF_DW + H], p[OFF_DB]


def forward(params, Ahat, sdinv, mask, r, bf16_ops=True):
    rnd = bf16 if bf16_ops else (lambda a: np.asarray(a, dtype=np.float64))
    E, eb, W, b, dw, db = unpack(params)
    t = np.asarray(r, dtype=np.float64) * sdinv
    s = np.sqrt(float(t @ t) / len(t))
    x0 = (t * (1.0 / s if s > 0 else 0.0)).astype(np.float32).astype(np.float64)
    ax0 = Ahat @ x0
    Z0 = np.outer(x0, E[:, 0]) + np.outer(ax0, E[:, 1]) + eb
    Hs = [np.maximum(Z0, 0.0)]
    Ys = [None]
    for l in range(LAYERS):
        Y = Ahat @ Hs[-1]
        X = np.concatenate([Hs[-1], Y], axis=1)
        Z = rnd(X) @ rnd(W[l]).T + b[l]
        Ys.append(Y)
        Hs.append(np.maximum(Z, 0.0))
    free = ~np.asarray(mask, dtype=bool)
    yhat = x0 + np.where(free, Hs[-1] @ dw + db, 0.0)
    return dict(s=s, x0=x0, ax0=ax0, H=Hs, Y=Ys, yhat=yhat)


def apply(params, Ahat, sdinv, mask, r, bf16_ops=True):
    f = forward(params, Ahat, sdinv, mask, r, bf16_ops)
    return f["s"] * sdinv * f["yhat"]


def apply_inference(params, Ahat, sdinv, mask, r):
    """M(r) as the inference kernels compute it: rhat = D^-1/2 r in float32
    scaled by float32(1/s) after the aggregation, activations stored in BF16
    (H0..H2 rounded after the relu), aggregation of the stored values in
    float, the last layer's relu output fed to the decoder unrounded."""
    E, eb, W, b, dw, db = unpack(params)
    t = np.asarray(r, dtype=np.float64) * sdinv
    s = np.sqrt(float(t @ t) / len(t))
    f32 = np.float32
    rhat = t.astype(f32)
    inv = f32(1.0 / s if s > 0 else 0.0)
    x0 = (rhat * inv).astype(np.float64)
    ax0 = ((Ahat @ rhat.astype(np.float64)).astype(f32) * inv).astype(np.float64)
    Hc = bf16(np.maximum(np.outer(x0, E[:, 0]) + np.outer(ax0, E[:, 1]) + eb, 0.0))
    for l in range(LAYERS):
        Y = Ahat @ Hc
        Z = np.concatenate([Hc, bf16(Y)], axis=1) @ bf16(W[l]).T + b[l]
        Hc = np.maximum(Z, 0.0)
        if l + 1 < LAYERS:
            Hc = bf16(Hc)
    free = ~np.asarray(mask, dtype=bool)
    yhat = x0 + np.where(free, Hc @ dw + db, 0.0)
    return s * sdinv * yhat


def loss_grad(params, Ahat, sdinv, mask, r, e, bf16_ops=True):
    """(loss, gradient) for one residual/error pair."""
    rnd = bf16 if bf16_ops else (lambda a: np.asarray(a, dtype=np.float64))
    E, eb, W, b, dw, db = unpack(params)
    f = forward(params, Ahat, sdinv, mask, r, bf16_ops)
    s = f["s"]
    N = len(f["yhat"])
    tgt = np.asarray(e, dtype=np.float64) / sdinv / s
    d = f["yhat"] - tgt
    q = Ahat @ d
    loss = float(d @ q) / N
    g = np.where(np.asarray(mask, dtype=bool), 0.0, 2.0 * q / N)
    G = np.zeros(NPARAM)
    Hs, Ys = f["H"], f["Y"]
    G[OFF_DW:OFF_DW + H] = Hs[LAYERS].T @ g
    G[OFF_DB] = g.sum()
    dH = np.outer(g, dw)
    for l in range(LAYERS, 0, -1):
        dZ = dH * (Hs[l] > 0)
        X = np.concatenate([Hs[l - 1], Ys[l]], axis=1)
        o = OFF_L + (l - 1) * LSZ
        G[o:o + H * 2 * H] = (rnd(dZ).T @ rnd(X)).ravel()
        G[o + H * 2 * H:o + LSZ] = dZ.sum(axis=0)
        dX = rnd(dZ) @ rnd(W[l - 1])
        dH = dX[:, :H] + Ahat.T @ dX[:, H:]
    dZ0 = dH * (Hs[0] > 0)
    G[OFF_EW:OFF_EW + 2 * H] = np.stack([dZ0.T @ f["x0"], dZ0.T @ f["ax0"]], axis=1).ravel()
    G[OFF_EB:OFF_EB + H] = dZ0.sum(axis=0)
    return loss, G


def init_params(seed, decoder_scale=0.0):
    """A parameter vector with the GPU initialiser's distribution (not its
    values): He-normal layers, small positive biases, decoder scaled by
    decoder_scale."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    p[OFF_EW:OFF_EW + 2 * H] = rng.standard_normal(2 * H) * 0.7
    p[OFF_EB:OFF_EB + H] = 0.05
    for l in range(LAYERS):
        o = OFF_L + l * LSZ
        p[o:o + H * 2 * H] = rng.standard_normal(H * 2 * H) * np.sqrt(2.0 / (2 * H))
        p[o + H * 2 * H:o + LSZ] = 0.01 * rng.standard_normal(H)
    p[OFF_DW:OFF_DW + H] = decoder_scale * rng.standard_normal(H)
    p[OFF_DB] = 0.01 * decoder_scale
    return p
