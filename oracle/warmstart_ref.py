"""CPU reference of the warm-start network (forward, loss, backward).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels in
samos_b200/csrc/sg_ml.cu; only tests/ import it.  The network has no
counterpart in the reference code (the learned part is new), so this file
restates the network's own definition:

  e_ij  = (r, a_i, a_j, a_i + a_j - r)            for r = |d_ij| < rc
  s_i   = sum_j relu(W1a e_ij + b1a)
  h_i   = relu(s_i W1b + b1b)
  [P|Q] = h Wpq
  w_ij  = relu(P_i + Q_j + W2e e_ij + b2) . w2 + c
  disp_i = sum_j w_ij d_ij / r_ij
  loss  = sum_i |disp_i - t_i|^2 / n

Arithmetic is float64.  With ``bf16=True`` the tensors that the CUDA path
stores in BF16 (s, h, the GEMM weights, the GEMM operands of the backward
pass) are rounded to BF16 (round to nearest even) at the same points, and
the BF16 rounding of s is passed straight through in the backward pass, as
the CUDA path does.  With ``bf16=False`` the network is exact float64, which
the finite-difference test uses.
"""
from __future__ import annotations

import numpy as np

F = 64
OFF = dict(W1a=(0, (64, 4)), b1a=(256, (64,)), W1b=(320, (64, 64)), b1b=(4416, (64,)), Wpq=(4480, (64, 128)),
           b2=(12672, (64,)), W2e=(12736, (64, 4)), w2=(12992, (64,)), c=(13056, (1,)))
NPARAM = 13057


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round float values to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray) -> dict:
    return {k: np.asarray(p[o:o + int(np.prod(s))], np.float64).reshape(s) for k, (o, s) in OFF.items()}


def edges(x, y, radius, L, rc):
    """All ordered pairs (i, j), i != j, with minimum-image distance r < rc.
    Returns i, j, e [E, 4] (features as float32 values), u [E, 2]."""
    n = len(x)
    I, J = np.nonzero(~np.eye(n, dtype=bool))
    dx = x[J] - x[I]
    dy = y[J] - y[I]
    dx = np.where(dx > 0.5 * L, dx - L, np.where(dx < -0.5 * L, dx + L, dx))
    dy = np.where(dy > 0.5 * L, dy - L, np.where(dy < -0.5 * L, dy + L, dy))
    r = np.sqrt(dx * dx + dy * dy)
    keep = (r < rc) & (r > 0)
    I, J, dx, dy, r = I[keep], J[keep], dx[keep], dy[keep], r[keep]
    a = radius.astype(np.float32).astype(np.float64)
    rf = r.astype(np.float32).astype(np.float64)
    e = np.stack([rf, a[I], a[J], (a[I] + a[J] - rf).astype(np.float32)], axis=1)
    u = np.stack([(dx / r).astype(np.float32), (dy / r).astype(np.float32)], axis=1).astype(np.float64)
    return I, J, e, u


class Net:
    def __init__(self, params: np.ndarray, bf16: bool = True):
        self.W = unpack(params)
        self.bf16 = bf16

    def _q(self, a):
        return bf16_round(a) if self.bf16 else np.asarray(a, np.float64)

    def forward(self, n, I, J, e, u):
        W, q = self.W, self._q
        z1 = e @ W["W1a"].T + W["b1a"]
        s = np.zeros((n, F))
        np.add.at(s, I, np.maximum(z1, 0.0))
        s16 = q(s)
        h = q(np.maximum(s16 @ q(W["W1b"]) + W["b1b"], 0.0))
        PQ = h @ q(W["Wpq"])
        if self.bf16:
            PQ = PQ.astype(np.float32).astype(np.float64)
        z2 = PQ[I, :F] + PQ[J, F:] + e @ W["W2e"].T + W["b2"]
        a2 = np.maximum(z2, 0.0)
        w = a2 @ W["w2"] + W["c"][0]
        disp = np.zeros((n, 2))
        np.add.at(disp, I, w[:, None] * u)
        self.cache = dict(n=n, I=I, J=J, e=e, u=u, z1=z1, s16=s16, h=h, PQ=PQ, z2=z2, a2=a2)
        return disp

    def loss_and_grad(self, n, I, J, e, u, target, inv_n):
        W, q = self.W, self._q
        disp = self.forward(n, I, J, e, u)
        c = self.cache
        d = disp - target
        loss = float(np.sum(d * d)) * inv_n
        gd = 2.0 * d * inv_n
        gw = np.sum(gd[I] * u, axis=1)
        g = {k: np.zeros_like(v) for k, v in W.items()}
        g["w2"] = c["a2"].T @ gw
        g["c"] = np.array([gw.sum()])
        gz2 = (c["z2"] > 0) * (gw[:, None] * W["w2"][None, :])
        g["b2"] = gz2.sum(0)
        g["W2e"] = gz2.T @ e
        gPQ = np.zeros((n, 2 * F))
        np.add.at(gPQ[:, :F], I, gz2)
        np.add.at(gPQ[:, F:], J, gz2)
        gPQ16 = q(gPQ)
        g["Wpq"] = c["h"].T @ gPQ16
        gh = gPQ16 @ q(W["Wpq"]).T
        if self.bf16:
            gh = gh.astype(np.float32).astype(np.float64)
        gpre = q(gh * (c["h"] > 0))
        g["b1b"] = gpre.sum(0)
        g["W1b"] = c["s16"].T @ gpre
        gs = gpre @ q(W["W1b"]).T
        gz1 = (c["z1"] > 0) * gs[I]
        g["b1a"] = gz1.sum(0)
        g["W1a"] = gz1.T @ e
        flat = np.zeros(NPARAM)
        for k, (o, s) in OFF.items():
            flat[o:o + int(np.prod(s))] = g[k].reshape(-1)
        return loss, disp, flat


def loss_only(params, n, I, J, e, u, target, inv_n, bf16=False):
    net = Net(params, bf16=bf16)
    d = net.forward(n, I, J, e, u) - target
    return float(np.sum(d * d)) * inv_n
