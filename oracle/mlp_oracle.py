"""FP64 numpy restatement of the radiation surrogate's network, for tests only.

TEST INFRASTRUCTURE ONLY: the parity checker for libexotx's MLP kernels
(exotx_mlp_forward / exotx_mlp_backward / exotx_mlp_adam).  The surrogate has
no counterpart in the reference, so this file restates the textbook maths the
kernels implement:
  hidden layer  z = h W^T + b,  h' = silu(z) = z / (1 + e^-z)
  output layer  y = h W^T + b
  loss          mean over rows and outputs of (y - t)^2
  backward      dW = dz^T h, db = sum_rows dz, dh = dz W, dz = dh * silu'(z)
  Adam          m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
                p -= lr (m / (1-b1^t)) / (sqrt(v / (1-b2^t)) + eps)
Parameters use the library's flat layout: per layer W (dout x din), then b.
"""
import numpy as np


def unpack(params, layers):
    out = []
    for wo, bo, di, do in layers:
        out.append((params[wo:wo + di * do].reshape(do, di), params[bo:bo + do]))
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, layers, X):
    P = unpack(np.asarray(params, np.float64), layers)
    h = np.asarray(X, np.float64)
    zs, hs = [], [h]
    for l, (W, b) in enumerate(P):
        z = h @ W.T + b
        zs.append(z)
        if l < len(P) - 1:
            h = silu(z)
            hs.append(h)
        else:
            h = z
    return h, zs, hs


def loss_and_grads(params, layers, X, T, W=None):
    """Mean squared error (each element's squared error weighted by W when
    given) and its gradient in the flat parameter layout."""
    params = np.asarray(params, np.float64)
    P = unpack(params, layers)
    Y, zs, hs = forward(params, layers, X)
    n = Y.size
    d = Y - np.asarray(T, np.float64)
    w = np.ones_like(d) if W is None else np.asarray(W, np.float64)
    loss = float((w * d * d).sum() / n)
    dz = 2.0 * w * d / n
    g = np.zeros_like(params)
    for l in range(len(P) - 1, -1, -1):
        wo, bo, di, do = layers[l]
        W, _ = P[l]
        g[wo:wo + di * do] = (dz.T @ hs[l]).ravel()
        g[bo:bo + do] = dz.sum(0)
        if l > 0:
            dz = (dz @ W) * silu_grad(zs[l - 1])
    return loss, g


def adam(params, grads, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grads
    v = b2 * v + (1 - b2) * grads * grads
    p = params - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
