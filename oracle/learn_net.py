"""CPU restatement of the learned refinement predictor (test infrastructure).

The predictor has no counterpart in the reference (its only refinement
criteria are the plain vorticity / Q rules, solver_lbm_criterion.cu); this
module states the network the CUDA library trains and evaluates, in numpy,
so that the library's forward pass, loss and gradients can be checked:

  per block of P = 4^d cells, zero padding at the block faces,
  h1 = relu(conv3^d(x0; 8 -> 32) + b1)
  h2 = relu(conv3^d(h1; 32 -> 32) + b2)
  z  = mean over cells of conv3^d(h2; 32 -> 2) + b3
  loss = sum_j wt_j sum_k (pw_k y_jk softplus(-z_jk) + (1 - y_jk) softplus(z_jk))
         / (2 sum_j wt_j)          (pw: positive-class weights of the outputs)

Parameters are one flat FP32 vector: W1 [32][K1p] (K1 = 8T real columns,
zero padding up to a multiple of 16), b1 [32], W2 [32][32T], b2 [32],
W3 [2][32T], b3 [2]; T = 3^d taps, tap = (dx+1) + 3(dy+1) + 9(dz+1), im2col
column = tap * channels + channel.

With ``bf16=True`` the operands are rounded to BF16 (round to nearest even)
at the points where the CUDA path feeds its tensor-core GEMMs: the im2col
columns and weights of every layer, the pooled-loss gradient, and the
post-ReLU gradients of the hidden layers; sums and bias gradients stay in
high precision.  With ``bf16=False`` the same network is exact in FP64,
which ``finite_difference`` checks.

Only tests import this module; the library never calls it.
"""
from __future__ import annotations

import numpy as np

C0, CH, NO = 8, 32, 2


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u.astype(np.uint64) + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.view(np.float32)


def geometry(dim):
    P, T = (16, 9) if dim == 2 else (64, 27)
    K1 = T * C0
    K1p = (K1 + 15) // 16 * 16
    return P, T, K1, K1p, T * CH


def tap_table(dim):
    """nbr[c, t] = cell reached from cell c along tap t, P (a zero row) outside."""
    P, T = geometry(dim)[:2]
    nbr = np.full((P, T), P, dtype=np.int64)
    for c in range(P):
        I, J, K = c & 3, (c >> 2) & 3, (c >> 4) if dim == 3 else 0
        for t in range(T):
            dx, dy, dz = t % 3 - 1, (t // 3) % 3 - 1, (t // 9 - 1) if dim == 3 else 0
            i, j, k = I + dx, J + dy, K + dz
            if 0 <= i <= 3 and 0 <= j <= 3 and 0 <= k <= 3:
                nbr[c, t] = i + 4 * j + 16 * k
    return nbr


def split(w, dim):
    P, T, K1, K1p, K2 = geometry(dim)
    o = 0
    out = {}
    for name, shape in (("W1", (CH, K1p)), ("b1", (CH,)), ("W2", (CH, K2)), ("b2", (CH,)), ("W3", (NO, K2)),
                        ("b3", (NO,))):
        n = int(np.prod(shape))
        out[name] = np.asarray(w[o:o + n]).reshape(shape)
        o += n
    assert o == len(w)
    return out


def im2col(H, dim, n, kp=None):
    """H [n*P][C] -> [n*P][kp] (column = tap * C + channel, zero outside the block)."""
    P, T = geometry(dim)[:2]
    C = H.shape[1]
    Hp = np.concatenate([H.reshape(n, P, C), np.zeros((n, 1, C), H.dtype)], axis=1)
    X = Hp[:, tap_table(dim), :].reshape(n * P, T * C)
    if kp is not None and kp > T * C:
        X = np.concatenate([X, np.zeros((n * P, kp - T * C), X.dtype)], axis=1)
    return X


def col2im(dX, dim, n, C):
    """Adjoint of im2col: dH[n*P][C] from dX [n*P][>= T*C]."""
    P, T = geometry(dim)[:2]
    nbr = tap_table(dim)
    d = dX[:, :T * C].reshape(n, P, T, C)
    dH = np.zeros((n, P + 1, C), dX.dtype)
    for t in range(T):
        np.add.at(dH, (slice(None), nbr[:, t], slice(None)), d[:, :, t, :])
    return dH[:, :P, :].reshape(n * P, C)


def forward_backward(w, X0, dim, Y=None, Wt=None, bf16_emulation=True, pos_weight=(1.0, 1.0)):
    """Logits [n][2]; with labels also (loss, flat gradient).  X0 [n*P][8]."""
    P, T, K1, K1p, K2 = geometry(dim)
    n = X0.shape[0] // P
    f = np.float64
    r = (lambda a: bf16(a).astype(f)) if bf16_emulation else (lambda a: np.asarray(a, f))
    p = split(np.asarray(w, np.float32 if bf16_emulation else f), dim)
    W1, W2, W3 = r(p["W1"]), r(p["W2"]), r(p["W3"])
    b1, b2, b3 = (p[k].astype(f) for k in ("b1", "b2", "b3"))
    hold = (lambda a: a.astype(np.float32).astype(f)) if bf16_emulation else (lambda a: a)

    X1 = r(im2col(np.asarray(X0, f), dim, n, K1p))
    H1 = hold(np.maximum(hold(X1 @ W1.T) + b1, 0.0))
    X2 = r(im2col(H1, dim, n))
    H2 = hold(np.maximum(hold(X2 @ W2.T) + b2, 0.0))
    X3 = r(im2col(H2, dim, n))
    Z = hold(X3 @ W3.T)
    z = Z.reshape(n, P, NO).mean(axis=1) + b3
    if Y is None:
        return z
    Y = np.asarray(Y, f)
    Wt = np.asarray(Wt, f)
    cnt = Wt.sum()
    inv = 1.0 / (cnt * NO) if cnt > 0 else 0.0
    pw = np.asarray(pos_weight, f)[None, :]
    sp = np.log1p(np.exp(-np.abs(z)))
    loss = float((Wt[:, None] * (pw * Y * (np.maximum(-z, 0) + sp) + (1 - Y) * (np.maximum(z, 0) + sp))).sum() * inv)
    s = 1.0 / (1.0 + np.exp(-z))
    g = Wt[:, None] * (s * (pw * Y + 1 - Y) - pw * Y) * inv           # dL/dz [n][2]
    db3 = g.sum(axis=0)
    dZ = r(np.repeat(g / P, P, axis=0))                                 # [n*P][2]
    dW3 = dZ.T @ X3
    dH2 = col2im(dZ @ W3, dim, n, CH)
    dY2 = np.where(H2 > 0, dH2, 0.0)
    db2 = dY2.sum(axis=0)
    dY2r = r(dY2)
    dW2 = dY2r.T @ X2
    dH1 = col2im(dY2r @ W2, dim, n, CH)
    dY1 = np.where(H1 > 0, dH1, 0.0)
    db1 = dY1.sum(axis=0)
    dW1 = r(dY1).T @ X1
    dW1[:, K1:] = 0.0
    grad = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return z, loss, grad


def finite_difference(w, X0, dim, Y, Wt, idx, h=1e-6, pos_weight=(1.0, 1.0)):
    """Central differences of the exact (FP64) loss at parameter indices idx."""
    w = np.asarray(w, np.float64)
    out = []
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        lp = forward_backward(wp, X0, dim, Y, Wt, bf16_emulation=False, pos_weight=pos_weight)[1]
        lm = forward_backward(wm, X0, dim, Y, Wt, bf16_emulation=False, pos_weight=pos_weight)[1]
        out.append((lp - lm) / (2 * h))
    return np.array(out)


def init_params(dim, seed):
    """He-uniform weights (padding columns of W1 zero), zero biases - the
    distribution the library draws from, not its exact values."""
    P, T, K1, K1p, K2 = geometry(dim)
    rng = np.random.default_rng(seed)
    parts = []
    for nout, k, kp in ((CH, K1, K1p), (CH, K2, K2), (NO, K2, K2)):
        a = np.sqrt(6.0 / k)
        W = np.zeros((nout, kp))
        W[:, :k] = rng.uniform(-a, a, (nout, k))
        parts += [W.ravel(), np.zeros(nout)]
    return np.concatenate(parts)
