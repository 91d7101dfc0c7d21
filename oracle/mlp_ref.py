"""CPU reference of the cost-model MLP (TEST INFRASTRUCTURE ONLY).

Float64 numpy restatement of the network libots trains on the GPU
(ics-12-overlapped-tiling_b200/csrc/ots_mlp.cu): inputs standardised as
(x - mean) * inv_std, [Linear -> SiLU] x (layers - 1) -> Linear, mean
squared error on standardised targets.  Parameters are laid out layer by
layer as W (out x in, row-major) then b (out).  Used to check the CUDA
forward/backward pass; its own backward pass is checked against finite
differences.
"""
import numpy as np


def layer_dims(n_in, hidden, layers):
    return [n_in] + [hidden] * (layers - 1) + [1]


def unpack(params, dims):
    out, off = [], 0
    for i, o in zip(dims[:-1], dims[1:]):
        W = params[off:off + i * o].reshape(o, i)
        off += i * o
        b = params[off:off + o]
        off += o
        out.append((W, b))
    assert off == len(params)
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(X, params, dims, mean, inv_std):
    A = (np.asarray(X, np.float64) - mean) * inv_std
    cache = []
    layers = unpack(np.asarray(params, np.float64), dims)
    for li, (W, b) in enumerate(layers):
        Z = A @ W.T + b
        cache.append((A, Z))
        A = Z if li == len(layers) - 1 else silu(Z)
    return A[:, 0], cache, layers


def loss_grad(X, y, params, dims, mean, inv_std, y_mean, y_std):
    p, cache, layers = forward(X, params, dims, mean, inv_std)
    t = (np.asarray(y, np.float64) - y_mean) / y_std
    B = len(t)
    d = p - t
    loss = float(np.mean(d * d))
    dZ = (2.0 * d / B)[:, None]
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        A_in, Z = cache[li]
        W, _ = layers[li]
        gW = dZ.T @ A_in
        gb = dZ.sum(axis=0)
        grads[li] = (gW, gb)
        if li > 0:
            dA = dZ @ W
            dZ = dA * dsilu(cache[li - 1][1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
