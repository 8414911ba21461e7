"""NumPy FP32 restatement of the surrogate network and its training step (TEST INFRASTRUCTURE
ONLY: the checker of the device's tcgen05 forward and backward kernels, never the product).

The network and its loss are this project's own (the reference has no surrogate): a 1280 ->
128 -> 128 -> 1 perceptron with SiLU activations.  The device rounds to BF16 at fixed points
-- the inputs and weights it reads, the first hidden activation (the second layer's operand),
and the gradients that feed a tensor-core product (dz2, dz1, and h1 for dW2) -- and accumulates
in FP32; this restatement rounds at the same points, so the two agree to FP32 summation order.
"""

from __future__ import annotations

import numpy as np

IN, H = 1280, 128


def bf16(a):
    """Round float32 to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(a):
    """The BF16 bit patterns (uint16) of float32 values rounded to nearest even."""
    return (bf16(a).view(np.uint32) >> 16).astype(np.uint16)


def sigm(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * sigm(z)


def dsilu(z):
    s = sigm(z)
    return s * (1.0 + z * (1.0 - s))


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    p = dict(w1=(rng.standard_normal((H, IN)) / np.sqrt(IN)).astype(np.float32),
             b1=np.zeros(H, np.float32),
             w2=(rng.standard_normal((H, H)) / np.sqrt(H)).astype(np.float32),
             b2=np.zeros(H, np.float32),
             w3=(rng.standard_normal(H) / np.sqrt(H)).astype(np.float32),
             b3=np.zeros(1, np.float32))
    return p


def forward(p, x):
    """y for rows x (float32, already BF16 values), with the device's rounding points."""
    x = bf16(x).astype(np.float64)
    z1 = x @ bf16(p["w1"]).astype(np.float64).T + p["b1"]
    h1 = bf16(silu(z1).astype(np.float32)).astype(np.float64)
    z2 = h1 @ bf16(p["w2"]).astype(np.float64).T + p["b2"]
    h2 = silu(z2)
    y = h2 @ p["w3"].astype(np.float64) + float(p["b3"][0])
    return y.astype(np.float32), dict(z1=z1, h1=h1, z2=z2, h2=h2)


def grads(p, x, target):
    """Loss (sum of squared pair errors) and gradients of the mean pair loss, rows in pairs
    (2q, 2q+1) whose antisymmetric part (y0 - y1)/2 is fitted to target[q]."""
    y, c = forward(p, x)
    y = y.astype(np.float64)
    npair = x.shape[0] // 2
    s = 0.5 * (y[0::2] - y[1::2])
    diff = s - target.astype(np.float64)
    loss = float(np.sum(diff * diff))
    gy = np.zeros_like(y)
    gy[0::2] = diff / npair
    gy[1::2] = -diff / npair
    dw3 = c["h2"].T @ gy
    db3 = np.array([gy.sum()])
    dz2 = gy[:, None] * p["w3"][None, :].astype(np.float64) * dsilu(c["z2"])
    db2 = dz2.sum(axis=0)
    dz2b = bf16(dz2.astype(np.float32)).astype(np.float64)
    dw2 = dz2b.T @ c["h1"]
    dh1 = dz2b @ bf16(p["w2"]).astype(np.float64)
    dz1 = dh1 * dsilu(c["z1"])
    db1 = dz1.sum(axis=0)
    dz1b = bf16(dz1.astype(np.float32)).astype(np.float64)
    dw1 = dz1b.T @ bf16(x).astype(np.float64)
    return loss, dict(w1=dw1, b1=db1, w2=dw2, b2=db2, w3=dw3, b3=db3)


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step in place (bias-corrected), as the device's optimiser kernel."""
    c1 = 1.0 / (1.0 - b1 ** step)
    c2 = 1.0 / (1.0 - b2 ** step)
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] * g[k]
        p[k] = (p[k] - lr * (m[k] * c1) / (np.sqrt(v[k] * c2) + eps)).astype(np.float32)
