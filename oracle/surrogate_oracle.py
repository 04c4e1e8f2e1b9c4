"""CPU oracle of the convolutional neural operator (TEST INFRASTRUCTURE, not product code).

Only ``tests/`` use this module, as the checker of the surrogate's CUDA kernels
(torchfdtd_b200/csrc/surrogate.cu). It restates in NumPy the same network: packed input (2 rho - 1, x, y, 1,
zeros to 16 channels), 8 conv layers (3x3, zero padding 1, stride 1/2 alternating, 64 channels, GELU in its
tanh form), a linear head on the flattened last feature map and the mean-squared loss, with forward and
backward passes.

``bf16=True`` rounds what the kernels hold in BF16 (packed input, weights, pre-activations, activations and
the back-propagated pre-activation gradients) to bfloat16 (round to nearest even) and accumulates in
float64, so the GPU results agree to accumulation-order rounding; ``bf16=False`` is the exact float64
network that finite differences check.
"""
from __future__ import annotations

import numpy as np

LAYERS = ((16, 1), (64, 2), (64, 1), (64, 2), (64, 1), (64, 2), (64, 1), (64, 2))
C = 0.7978845608028654


def to_bf16(x):
    """Round float values to bfloat16 (nearest even) and return them as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1 + np.tanh(C * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    th = np.tanh(C * (z + 0.044715 * z ** 3))
    return 0.5 * (1 + th) + 0.5 * z * (1 - th * th) * C * (1 + 3 * 0.044715 * z * z)


def pack_input(rho):
    n, h, w = rho.shape
    x = np.zeros((n, h, w, 16))
    x[..., 0] = 2 * rho - 1
    x[..., 1] = np.linspace(-1, 1, w)[None, None, :] if w > 1 else 0
    x[..., 2] = np.linspace(-1, 1, h)[None, :, None] if h > 1 else 0
    x[..., 3] = 1
    return x


def out_size(n, stride):
    return (n - 1) // stride + 1


def conv(x, w, b, stride):
    """x (n, h, w, ci), w (9, co, ci), b (co,) -> z (n, ho, wo, co)."""
    n, h, wd, ci = x.shape
    ho, wo = out_size(h, stride), out_size(wd, stride)
    xp = np.zeros((n, h + 2, wd + 2, ci))
    xp[:, 1:-1, 1:-1] = x
    z = np.zeros((n, ho, wo, w.shape[1])) + b
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        patch = xp[:, ky:ky + (ho - 1) * stride + 1:stride, kx:kx + (wo - 1) * stride + 1:stride]
        z += patch @ w[tap].T
    return z


def conv_dgrad(dz, w, shape, stride):
    n, h, wd, ci = shape
    ho, wo = dz.shape[1:3]
    dxp = np.zeros((n, h + 2, wd + 2, ci))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        dxp[:, ky:ky + (ho - 1) * stride + 1:stride, kx:kx + (wo - 1) * stride + 1:stride] += dz @ w[tap]
    return dxp[:, 1:-1, 1:-1]


def conv_wgrad(dz, x, stride):
    n, h, wd, ci = x.shape
    ho, wo = dz.shape[1:3]
    xp = np.zeros((n, h + 2, wd + 2, ci))
    xp[:, 1:-1, 1:-1] = x
    dw = np.zeros((9, dz.shape[3], ci))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        patch = xp[:, ky:ky + (ho - 1) * stride + 1:stride, kx:kx + (wo - 1) * stride + 1:stride]
        dw[tap] = dz.reshape(-1, dz.shape[3]).T @ patch.reshape(-1, ci)
    return dw, dz.sum(axis=(0, 1, 2))


class NetworkOracle:
    def __init__(self, params, bf16=True):
        """params: dict w0..w7 (9, 64, ci), b0..b7 (64,), wh (k, features), bh (k,)."""
        self.p = {k: np.asarray(v, dtype=np.float64) for k, v in params.items()}
        self.bf16 = bf16

    def _r(self, x):
        return to_bf16(x) if self.bf16 else x

    def forward(self, rho):
        x = self._r(pack_input(np.asarray(rho, dtype=np.float64)))
        self.xs, self.zs = [], []
        for l, (ci, stride) in enumerate(LAYERS):
            self.xs.append(x)
            z = conv(x, self._r(self.p[f'w{l}']), self.p[f'b{l}'], stride)
            zr = self._r(z)
            self.zs.append(zr)
            x = self._r(gelu(z))
        self.flat = x.reshape(x.shape[0], -1)
        return self.flat @ self.p['wh'].T + self.p['bh']

    def backward(self, dout, input_gradient=False):
        """Gradients of sum(dout * out) for every parameter (and d/d rho)."""
        g = {}
        g['wh'] = dout.T @ self.flat
        g['bh'] = dout.sum(axis=0)
        z = self.zs[-1]
        dflat = (dout @ self.p['wh']).reshape(z.shape)
        dz = self._r(dflat * gelu_grad(z))
        for l in range(len(LAYERS) - 1, -1, -1):
            ci, stride = LAYERS[l]
            g[f'w{l}'], g[f'b{l}'] = conv_wgrad(dz, self.xs[l], stride)
            if l > 0:
                dx = conv_dgrad(dz, self._r(self.p[f'w{l}']), self.xs[l].shape, stride)
                dz = self._r(dx * gelu_grad(self.zs[l - 1]))
            elif input_gradient:
                dx = conv_dgrad(dz, self._r(self.p[f'w{l}']), self.xs[l].shape, stride)
                g['rho'] = 2 * dx[..., 0]
        return g
