"""CPU restatement of the learned selector's network, its gradient and Adam.

TEST INFRASTRUCTURE ONLY: imported by tests/ to check the CUDA kernels
``fsb_mlp_forward`` / ``fsb_mlp_backward`` / ``fsb_adam_step``; the library
``flagsparse_public_b200`` never imports it.

FlagSparse has no learned selector (its launch parameters come from fixed
row-length buckets, spmm_csr.py:395-414, and device-property heuristics,
spmm_csr_opt_alg2.py:175-304), so there is no reference output to pin this
against; it is pinned instead by central finite differences of the loss
(``finite_difference_grad``) in the CPU tests.

Network: d_in -> h1 (ReLU) -> h2 (ReLU) -> d_out, parameters packed
W1[d_in][h1], b1[h1], W2[h1][h2], b2[h2], W3[h2][d_out], b3[d_out].
Loss: inv_terms * sum(mask * (Y - T)^2).  Computed in float64.
"""

import numpy as np


def unpack(params, d_in, h1, h2, d_out):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    shapes = [(d_in, h1), (h1,), (h1, h2), (h2,), (h2, d_out), (d_out,)]
    out = []
    for s in shapes:
        n = int(np.prod(s))
        out.append(p[o:o + n].reshape(s))
        o += n
    if o != p.size:
        raise ValueError(f"expected {o} parameters, got {p.size}")
    return out


def param_count(d_in, h1, h2, d_out):
    return d_in * h1 + h1 + h1 * h2 + h2 + h2 * d_out + d_out


def forward(X, params, dims):
    """Returns Y and the cache (Z1, Z2) of pre-activations."""
    W1, b1, W2, b2, W3, b3 = unpack(params, *dims)
    X = np.asarray(X, dtype=np.float64)
    Z1 = X @ W1 + b1
    H1 = np.maximum(Z1, 0.0)
    Z2 = H1 @ W2 + b2
    H2 = np.maximum(Z2, 0.0)
    Y = H2 @ W3 + b3
    return Y, (Z1, Z2)


def loss(X, params, dims, T, mask, inv_terms):
    Y, _ = forward(X, params, dims)
    return float(inv_terms * np.sum(np.asarray(mask) * (Y - np.asarray(T)) ** 2))


def backward(X, params, dims, T, mask, inv_terms):
    """Returns (grad packed like params, loss)."""
    W1, b1, W2, b2, W3, b3 = unpack(params, *dims)
    X = np.asarray(X, dtype=np.float64)
    Y, (Z1, Z2) = forward(X, params, dims)
    mask = np.asarray(mask, dtype=np.float64)
    diff = Y - np.asarray(T, dtype=np.float64)
    L = float(inv_terms * np.sum(mask * diff * diff))
    dY = 2.0 * diff * mask * inv_terms
    H2 = np.maximum(Z2, 0.0)
    H1 = np.maximum(Z1, 0.0)
    dW3 = H2.T @ dY
    db3 = dY.sum(0)
    dZ2 = (dY @ W3.T) * (Z2 > 0)
    dW2 = H1.T @ dZ2
    db2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2.T) * (Z1 > 0)
    dW1 = X.T @ dZ1
    db1 = dZ1.sum(0)
    g = np.concatenate([a.ravel() for a in (dW1, db1, dW2, db2, dW3, db3)])
    return g, L


def finite_difference_grad(X, params, dims, T, mask, inv_terms, h=1e-6):
    """Central differences of the loss (pins ``backward``)."""
    p = np.asarray(params, dtype=np.float64).copy()
    g = np.zeros_like(p)
    for i in range(p.size):
        old = p[i]
        p[i] = old + h
        lp = loss(X, p, dims, T, mask, inv_terms)
        p[i] = old - h
        lm = loss(X, p, dims, T, mask, inv_terms)
        p[i] = old
        g[i] = (lp - lm) / (2 * h)
    return g


def adam_step(params, grad, m1, m2, lr, beta1, beta2, eps, step, weight_decay=0.0):
    """One Adam step (Kingma & Ba 2015, bias-corrected); returns new (p, m1, m2)."""
    p = np.asarray(params, dtype=np.float64)
    g = np.asarray(grad, dtype=np.float64) + weight_decay * p
    m1 = beta1 * np.asarray(m1, dtype=np.float64) + (1 - beta1) * g
    m2 = beta2 * np.asarray(m2, dtype=np.float64) + (1 - beta2) * g * g
    bc1 = 1 - beta1 ** step
    bc2 = 1 - beta2 ** step
    p = p - lr * (m1 / bc1) / (np.sqrt(m2 / bc2) + eps)
    return p, m1, m2
