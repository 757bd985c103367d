"""CPU checker for the surrogate network kernels (test infrastructure only).

FP64 numpy forward/backward of the same network as cosenu_b200/csrc/mlp.cu:
layers W [out][in] (+ b), GELU (exact, erf form) between layers, loss
1/(rows*n_out) sum (y - t)^2, parameters flat per layer (W then b).  With
``emulate_bf16`` the values the GPU rounds to BF16 (input, weights, hidden
activations, layer gradients fed to the tensor cores) are rounded the same
way (round to nearest even), so the GPU gradients can be compared tightly;
without it the arithmetic is plain FP64 for the finite-difference check.
"""
from __future__ import annotations

import math

import numpy as np

_erf = np.vectorize(math.erf)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2 * math.pi)


class MLPOracle:
    def __init__(self, n_in: int, n_hidden: int, n_hidden_layers: int, n_out: int):
        self.n_in = n_in
        self.kpad = (n_in + 15) // 16 * 16
        self.din = [self.kpad] + [n_hidden] * n_hidden_layers
        self.dout = [n_hidden] * n_hidden_layers + [n_out]
        self.offsets = []
        off = 0
        for di, do in zip(self.din, self.dout):
            self.offsets.append((off, off + di * do))
            off += di * do + do
        self.nparam = off

    def unpack(self, theta):
        Ws, bs = [], []
        for (ow, ob), di, do in zip(self.offsets, self.din, self.dout):
            Ws.append(np.asarray(theta[ow:ow + di * do], dtype=np.float64).reshape(do, di))
            bs.append(np.asarray(theta[ob:ob + do], dtype=np.float64))
        return Ws, bs

    def forward(self, theta, x, emulate_bf16=False):
        Ws, bs = self.unpack(theta)
        r = (lambda a: bf16(a)) if emulate_bf16 else (lambda a: a)
        h = np.zeros((x.shape[0], self.kpad))
        h[:, :self.n_in] = x
        h = r(h)
        zs, hs = [], [h]
        for l, (W, b) in enumerate(zip(Ws, bs)):
            z = h @ r(W).T + b
            zs.append(z)
            if l < len(Ws) - 1:
                h = r(gelu(z))
                hs.append(h)
        return zs[-1], zs, hs

    def loss_grad(self, theta, x, t, emulate_bf16=False):
        Ws, bs = self.unpack(theta)
        r = (lambda a: bf16(a)) if emulate_bf16 else (lambda a: a)
        y, zs, hs = self.forward(theta, x, emulate_bf16)
        n = y.size
        loss = float(np.sum((y - t) ** 2) / n)
        dz = 2.0 * (y - t) / n
        grad = np.zeros(self.nparam)
        for l in range(len(Ws) - 1, -1, -1):
            ow, ob = self.offsets[l]
            dzr = r(dz)
            grad[ow:ow + Ws[l].size] = (dzr.T @ hs[l]).ravel()
            grad[ob:ob + bs[l].size] = dz.sum(axis=0)
            if l > 0:
                dh = dzr @ r(Ws[l])
                dz = dh * gelu_grad(zs[l - 1])
        return loss, grad
