"""ORACLE TEST INFRASTRUCTURE -- FP64 restatement of the warm-start network.

Not part of the shipped library: only tests/ import it, as the checker of
the device kernels in sparse-eigs-mex_b200/csrc/kernels/mpnn.cu (forward
pass, subspace loss and its gradient, backward pass).  Same parameter
layout as the device network: per layer l = 0 (input), 1..L (message
passing), L+1 (output) the weight matrix (rows = outputs, row-major) and
then the bias.
"""
from __future__ import annotations

import numpy as np


def layer_shapes(F, H, L, P):
    shapes = [(H, F)] + [(H, 2 * H)] * L + [(P, H)]
    return shapes


def unpack(params, F, H, L, P):
    out, off = [], 0
    for (o, i) in layer_shapes(F, H, L, P):
        W = params[off:off + o * i].reshape(o, i)
        off += o * i
        b = params[off:off + o]
        off += o
        out.append((W, b))
    return out


def forward(params, A, X, F, H, L, P):
    """A: scipy sparse (n x n) normalised adjacency; X: n x F.  Returns Y and the cache."""
    lay = unpack(params, F, H, L, P)
    W0, b0 = lay[0]
    h = np.tanh(X @ W0.T + b0)
    cache = [(X, None, h)]
    for l in range(1, L + 1):
        W, b = lay[l]
        m = A @ h
        x = np.concatenate([h, m], axis=1)
        hn = np.tanh(x @ W.T + b)
        cache.append((x, m, hn))
        h = hn
    Wo, bo = lay[L + 1]
    Y = h @ Wo.T + bo
    return Y, cache


def loss_and_dY(Y, U, eps=1e-8):
    """1 - trace(U^T P_Y U)/k and its gradient (the device uses the same
    regularisation eps * tr(G)/P of the Gram matrix)."""
    k = U.shape[1]
    P = Y.shape[1]
    G = Y.T @ Y
    G = G + eps * np.trace(G) / P * np.eye(P)
    B = Y.T @ U
    C = np.linalg.solve(G, B)
    loss = 1.0 - np.trace(B.T @ C) / k
    dY = -(2.0 / k) * (U - Y @ C) @ C.T
    return loss, dY


def backward(params, A, cache, dY, F, H, L, P):
    lay = unpack(params, F, H, L, P)
    grads = []
    Wo, bo = lay[L + 1]
    hL = cache[L][2]
    gWo = dY.T @ hL
    gbo = dY.sum(axis=0)
    dh = dY @ Wo
    for l in range(L, 0, -1):
        W, b = lay[l]
        x, m, hn = cache[l]
        dz = dh * (1.0 - hn ** 2)
        gW = dz.T @ x
        gb = dz.sum(axis=0)
        grads.append((gW, gb))
        dx = dz @ W
        dh = dx[:, :H] + A.T @ dx[:, H:]
    X, _, h0 = cache[0]
    W0, b0 = lay[0]
    dz = dh * (1.0 - h0 ** 2)
    g0 = (dz.T @ X, dz.sum(axis=0))
    ordered = [g0] + grads[::-1] + [(gWo, gbo)]
    return np.concatenate([np.concatenate([g.ravel(), gb]) for g, gb in ordered])
