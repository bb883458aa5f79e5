"""CPU oracle of the learned Cahn-Hilliard surrogate (numpy).

TEST INFRASTRUCTURE ONLY.  Restates the network the GPU kernels implement so
that tests can check the forward pass, the gradients and the mean-mass
projection.  The reference has no surrogate; this oracle is checked against
finite differences of itself in FP64 (tests/test_surrogate_oracle.py) and, in
the GPU tests, the tensor-core kernels are checked against it.

Network (one surrogate step = 50 FD time steps of CH):
    x0 = bf16((c - c_shift) * in_scale)                      [H, W, 1]
    z1 = conv3x3(x0, W1) + b1;  h1 = bf16(gelu(z1))           [H, W, 32]
    z2 = conv3x3(h1, W2) + b2;  h2 = bf16(gelu(z2))           [H, W, 32]
    z3 = conv3x3(h2, W3) + b3;  h3 = bf16(gelu(z3))           [H, W, 32]
    o  = conv3x3(h3, W4) + b4                                 [H, W, 1]
    c' = c + out_scale * o;  c' += mean(c) - mean(c')   (FP64 projection)
conv3x3 is a cross-correlation with circular padding; weights W[n, ky, kx, ci]
are BF16, accumulation FP32 (here FP64), gelu the tanh form
0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
"""
from __future__ import annotations

import numpy as np

CH = 32
LAYERS = ((1, CH), (CH, CH), (CH, CH), (CH, 1))  # (cin, cout)
GELU_K = np.sqrt(2.0 / np.pi)
GELU_C = 0.044715


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(GELU_K * (x + GELU_C * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_K * (x + GELU_C * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_K * (1.0 + 3.0 * GELU_C * x * x)


def conv3x3(x: np.ndarray, w: np.ndarray) -> np.ndarray:
    """x [B, H, W, ci], w [n, 3, 3, ci] -> [B, H, W, n], circular padding, FP64."""
    x = x.astype(np.float64)
    w = w.astype(np.float64)
    out = np.zeros(x.shape[:3] + (w.shape[0],))
    for ky in range(3):
        for kx in range(3):
            xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(1, 2))  # xs[y, x] = x[y + ky - 1, x + kx - 1]
            out += xs @ w[:, ky, kx, :].T
    return out


def conv3x3_wgrad(x: np.ndarray, dz: np.ndarray) -> np.ndarray:
    """dW[n, ky, kx, ci] = sum_p dz[p, n] x[p + (ky-1, kx-1), ci]."""
    x = x.astype(np.float64)
    dz = dz.astype(np.float64)
    n, ci = dz.shape[-1], x.shape[-1]
    dw = np.zeros((n, 3, 3, ci))
    for ky in range(3):
        for kx in range(3):
            xs = np.roll(x, shift=(1 - ky, 1 - kx), axis=(1, 2))
            dw[:, ky, kx, :] = np.einsum("bhwn,bhwc->nc", dz, xs)
    return dw


def conv3x3_dgrad(dz: np.ndarray, w: np.ndarray) -> np.ndarray:
    """dx[p, ci] = sum_{tap, n} dz[p - tap, n] w[n, tap, ci]."""
    dz = dz.astype(np.float64)
    w = w.astype(np.float64)
    dx = np.zeros(dz.shape[:3] + (w.shape[-1],))
    for ky in range(3):
        for kx in range(3):
            ds = np.roll(dz, shift=(ky - 1, kx - 1), axis=(1, 2))  # ds[y, x] = dz[y - ky + 1, x - kx + 1]
            dx += ds @ w[:, ky, kx, :]
    return dx


def init_params(seed: int = 0):
    """He-style init in FP32 (master copy); the kernels use bf16(W)."""
    rng = np.random.default_rng(seed)
    params = []
    for cin, cout in LAYERS:
        std = np.sqrt(2.0 / (9 * cin))
        w = rng.normal(0.0, std, size=(cout, 3, 3, cin)).astype(np.float32)
        b = np.zeros(cout, dtype=np.float32)
        params += [w, b]
    # last layer starts near zero so the untrained step is close to identity
    params[6] *= 0.1
    return params


def forward(params, c: np.ndarray, c_shift: float, in_scale: float):
    """c [B, H, W] -> (o [B, H, W], cache).  BF16 rounding where the kernels round."""
    W1, b1, W2, b2, W3, b3, W4, b4 = params
    x0 = bf16(((c - c_shift) * in_scale).astype(np.float32))[..., None]
    z1 = conv3x3(x0, bf16(W1)) + b1
    h1 = bf16(gelu(z1))
    z2 = conv3x3(h1, bf16(W2)) + b2
    h2 = bf16(gelu(z2))
    z3 = conv3x3(h2, bf16(W3)) + b3
    h3 = bf16(gelu(z3))
    o = (conv3x3(h3, bf16(W4)) + b4)[..., 0]
    return o, (x0, z1, h1, z2, h2, z3, h3)


def backward(params, cache, do: np.ndarray):
    """Gradients of sum(do * o) w.r.t. the eight parameter arrays (FP64)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = params
    x0, z1, h1, z2, h2, z3, h3 = cache
    dz4 = do[..., None].astype(np.float64)
    gW4 = conv3x3_wgrad(h3, dz4)
    gb4 = dz4.sum(axis=(0, 1, 2))
    dz3 = conv3x3_dgrad(dz4, bf16(W4)) * gelu_grad(z3)
    gW3 = conv3x3_wgrad(h2, dz3)
    gb3 = dz3.sum(axis=(0, 1, 2))
    dz2 = conv3x3_dgrad(dz3, bf16(W3)) * gelu_grad(z2)
    gW2 = conv3x3_wgrad(h1, dz2)
    gb2 = dz2.sum(axis=(0, 1, 2))
    dz1 = conv3x3_dgrad(dz2, bf16(W2)) * gelu_grad(z1)
    gW1 = conv3x3_wgrad(x0, dz1)
    gb1 = dz1.sum(axis=(0, 1, 2))
    return [gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4]


def mse_loss_and_grad(o: np.ndarray, target: np.ndarray):
    d = o.astype(np.float64) - target
    n = d.size
    return float((d * d).sum() / n), 2.0 * d / n


def step(params, c: np.ndarray, c_shift: float, in_scale: float, out_scale: float) -> np.ndarray:
    """One surrogate step with the FP64 mean-mass projection."""
    o, _ = forward(params, c[None], c_shift, in_scale)
    cn = c.astype(np.float64) + out_scale * o[0]
    cn += c.astype(np.float64).mean() - cn.mean()
    return cn
