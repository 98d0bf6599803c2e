"""CPU restatement of the learned face sensor (TEST INFRASTRUCTURE ONLY).

numpy FP64 forward/backward of the 21 -> 32 -> 32 -> 1 GELU (tanh form) network and of its
input features, used to check the GPU's BF16 tensor-core kernels (gradients,
logits) and the feature extraction.  No reference counterpart exists: the
sensor is an extension of the reference path, so this restatement is the
oracle for it (parity against it is "unpinned" by the reference).
"""
import math

import numpy as np

NF, NH, NP = 21, 32, 2145
OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3 = 0, 1024, 1056, 2080, 2112, 2144


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    W1 = w[OFF_W1:OFF_B1].reshape(32, 32)[:, :NF]
    return (W1, w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(32, 32), w[OFF_B2:OFF_W3],
            w[OFF_W3:OFF_B3], w[OFF_B3])


K0, K1 = math.sqrt(2.0 / math.pi), 0.044715


def gelu(x):
    """GELU in its tanh form (Hendrycks & Gimpel 2016), as the GPU evaluates it."""
    return 0.5 * x * (1.0 + np.tanh(K0 * (x + K1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(K0 * (x + K1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * K0 * (1.0 + 3.0 * K1 * x * x)


def forward(X, w):
    W1, b1, W2, b2, w3, b3 = unpack(w)
    z1 = X @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    return h2 @ w3 + b3, (z1, h1, z2, h2)


def loss_and_grad(X, y, w, pos_weight):
    """Mean BCE-with-logits (positive class weighted) and its gradient (NP floats)."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = X.shape[0]
    z, (z1, h1, z2, h2) = forward(X, w)
    sp_pos = np.logaddexp(0.0, -z)
    sp_neg = np.logaddexp(0.0, z)
    loss = np.mean(pos_weight * y * sp_pos + (1 - y) * sp_neg)
    sg = 1.0 / (1.0 + np.exp(-z))
    dz = (sg * (pos_weight * y + 1 - y) - pos_weight * y) / n
    g = np.zeros(NP)
    g[OFF_W3:OFF_B3] = h2.T @ dz
    g[OFF_B3] = dz.sum()
    dz2 = np.outer(dz, w3) * gelu_grad(z2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).ravel()
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    gW1 = np.zeros((32, 32))
    gW1[:, :NF] = dz1.T @ X
    g[OFF_W1:OFF_B1] = gW1.ravel()
    return loss, g


def weno_betas(a, b, c, d, e):
    t1, t2 = a - 2 * b + c, a - 4 * b + 3 * c
    b0 = 13.0 / 12.0 * t1 * t1 + 0.25 * t2 * t2
    t1, t2 = b - 2 * c + d, b - d
    b1 = 13.0 / 12.0 * t1 * t1 + 0.25 * t2 * t2
    t1, t2 = c - 2 * d + e, 3 * c - 4 * d + e
    b2 = 13.0 / 12.0 * t1 * t1 + 0.25 * t2 * t2
    return b0, b1, b2


def features(rho, p, un, gamma):
    """Features of faces from their 6-cell stencils: arrays of shape (n, 6)."""
    rho, p, un = (np.asarray(a, dtype=np.float64) for a in (rho, p, un))
    mr, mp, mu = rho.mean(1), p.mean(1), un.mean(1)
    cs = np.sqrt(np.maximum(gamma * mp / np.maximum(mr, 1e-30), 0.0))
    out = np.zeros((rho.shape[0], NF))
    for v, (X, m, sc) in enumerate([(rho, mr, 1e-3 * np.abs(mr)), (p, mp, 1e-3 * np.abs(mp)),
                                    (un, mu, 1e-3 * cs + 1e-30)]):
        d = X - m[:, None]
        mx = np.abs(d).max(1)
        out[:, 6 * v:6 * v + 6] = d / (mx + sc + 1e-30)[:, None]
    b0, b1, b2 = weno_betas(*(rho[:, s] for s in range(5)))
    den = b0 + b1 + b2 + (1e-3 * mr) ** 2 + 1e-30
    out[:, 18], out[:, 19], out[:, 20] = b0 / den, b1 / den, b2 / den
    return out


def stencils(W, d):
    """(rho, p, u_n) stencils of every face along axis d of a halo'd primitive field,
    in the device face order (face index fastest along k)."""
    g = 3
    nx, ny, nz = W.shape[0] - 6, W.shape[1] - 6, W.shape[2] - 6
    n = [nx, ny, nz]
    sl = []
    for s in range(6):
        idx = [slice(g, g + nx), slice(g, g + ny), slice(g, g + nz)]
        idx[d] = slice(s, s + n[d] + 1)
        sl.append(W[tuple(idx)])
    st = np.stack(sl, axis=-2)  # (..., 6, 5)
    st = st.reshape(-1, 6, 5)
    return st[:, :, 0], st[:, :, 1], st[:, :, 2 + d]
