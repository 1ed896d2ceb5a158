"""TEST INFRASTRUCTURE ONLY -- the oracle of the learned surrogate.

Float64 NumPy forward and backward of the control variate's network
(n_in -> H -> H -> H -> 1, GELU), with the same rounding points as the GPU
kernels (scp3_b200/csrc/mlp.cu): the weights of layers 0..2 and every layer's
input are rounded to BF16 before the product, accumulation is exact here (FP32
on the GPU), pre-activations and gradients are kept unrounded.  The reference
has no surrogate, so this oracle is project-defined; it pins the kernels'
gradients, not a reference behaviour.
"""
import numpy as np
from math import erf, sqrt, pi


def bf16(x):
    """Round-to-nearest-even to BF16, returned as float64."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / sqrt(2.0))) + z * np.exp(-0.5 * z * z) / sqrt(2.0 * pi)


def unpack(flat, n_in, hid):
    """Flat parameters (per layer: W out x in row-major, then b) -> lists."""
    shapes = [(hid, n_in), (hid, hid), (hid, hid), (1, hid)]
    W, B, k = [], [], 0
    for o, i in shapes:
        W.append(np.asarray(flat[k:k + o * i], dtype=np.float64).reshape(o, i))
        k += o * i
        B.append(np.asarray(flat[k:k + o], dtype=np.float64))
        k += o
    return W, B


def forward(flat, q, n_in, hid, scale=1.0, shift=0.0):
    W, B = unpack(flat, n_in, hid)
    h = np.asarray(q, dtype=np.float64)
    cache = []
    for l in range(3):
        x = bf16(h)
        z = x @ bf16(W[l]).T + B[l]
        cache.append((x, z))
        h = gelu(z)
    x = bf16(h)
    raw = x @ W[3][0] + B[3][0]
    return raw * scale + shift, (cache, x, raw)


def loss_and_grad(flat, q, t, n_in, hid, scale=1.0, shift=0.0):
    """MSE in raw units and its gradient, flat, in the kernels' order."""
    W, B = unpack(flat, n_in, hid)
    y, (cache, x3, raw) = forward(flat, q, n_in, hid, scale, shift)
    tr = (np.asarray(t, dtype=np.float64) - shift) / scale
    M = raw.size
    d = raw - tr
    loss = np.mean(d * d)
    dy = 2.0 * d / M
    grads_W, grads_B = [None] * 4, [None] * 4
    grads_W[3] = (dy @ x3)[None, :]
    grads_B[3] = np.array([dy.sum()])
    dh = np.outer(dy, W[3][0])
    for l in (2, 1, 0):
        x, z = cache[l]
        dz = dh * gelu_grad(z)
        grads_W[l] = dz.T @ x[:, :W[l].shape[1]]
        grads_B[l] = dz.sum(0)
        dh = dz @ W[l]
    flat_g = []
    for l in range(4):
        flat_g.append(grads_W[l].ravel())
        flat_g.append(grads_B[l].ravel())
    return loss, np.concatenate(flat_g)
