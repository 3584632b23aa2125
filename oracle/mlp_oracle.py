"""CPU oracle of the learned load-step predictor (test infrastructure only).

The predictor has no counterpart in the reference FAST code (cCtrlNR::Solver,
ctrl/ctrlnr.cpp:47-270, starts each load step from the last converged
displacements), so parity is unpinned against the reference; this module is
the project's own FP64 restatement, checked by finite differences:

* ``Mlp`` - the tanh network of the device predictor (hidden layers tanh,
  linear output, mean squared error), parameters laid out per layer as
  W [out][in] row-major then b [out];
* ``bf16`` - round-to-nearest-even to bfloat16, so ``Mlp(..., emulate=True)``
  reproduces the device arithmetic: every GEMM operand rounded to BF16,
  products accumulated exactly (FP64 here, FP32 on the device);
* ``pod_basis`` - the POD basis by a dense SVD of the snapshot matrix;
* ``samples`` - the training inputs and targets built from POD coefficients.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


class Mlp:
    def __init__(self, dims):
        self.dims = list(dims)

    def unpack(self, p):
        p = np.asarray(p, dtype=np.float64)
        out, off = [], 0
        for i, o in zip(self.dims[:-1], self.dims[1:]):
            W = p[off:off + o * i].reshape(o, i)
            off += o * i
            b = p[off:off + o]
            off += o
            out.append((W, b))
        assert off == p.size
        return out

    def forward(self, p, x, emulate=False):
        r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
        layers = self.unpack(p)
        hs = [np.asarray(x, dtype=np.float64)]
        for l, (W, b) in enumerate(layers):
            z = r(hs[-1]) @ r(W).T + b
            hs.append(np.tanh(z) if l + 1 < len(layers) else z)
        return hs

    def loss_grad(self, p, x, t, emulate=False):
        r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
        layers = self.unpack(p)
        hs = self.forward(p, x, emulate)
        y = hs[-1]
        t = np.asarray(t, dtype=np.float64)
        n = y.size
        loss = float(np.sum((y - t) ** 2) / n)
        g = 2.0 * (y - t) / n
        grads = [None] * len(layers)
        for l in range(len(layers) - 1, -1, -1):
            W, _ = layers[l]
            dW = r(g).T @ r(hs[l])
            db = g.sum(axis=0)
            grads[l] = (dW, db)
            if l > 0:
                g = (r(g) @ r(W)) * (1.0 - hs[l] ** 2)
        flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
        return loss, flat


def pod_basis(snapshots, k):
    """Left singular vectors of the [m][n] snapshot rows (n x k) and the
    captured energy fraction."""
    S = np.asarray(snapshots, dtype=np.float64)
    U, s, _ = np.linalg.svd(S.T, full_matrices=False)
    return U[:, :k], float(np.sum(s[:k] ** 2) / np.sum(s ** 2))


def samples(coef_by_traj, lam_by_traj, history, modes):
    """Training inputs/targets of the device predictor from POD coefficients
    (one [S][k] array per trajectory) and load factors, unscaled: per step
    s >= 2 the input [lambda_s, a_{s-1}, da_{s-1}, ..., da_{s-history+1}]
    (da_j = a_j - a_{j-1}, a_j = 0 for j <= 0) and the target
    da_s - rho da_{s-1}, rho = dlambda_s / dlambda_{s-1}."""
    X, T = [], []
    for A, lam in zip(coef_by_traj, lam_by_traj):
        A = np.asarray(A)
        k = A.shape[1]

        def a(s):
            return A[s - 1] if s >= 1 else np.zeros(k)

        def lm(s):
            return lam[s - 1] if s >= 1 else 0.0

        for s in range(2, len(lam) + 1):
            d1 = lm(s - 1) - lm(s - 2)
            rho = (lm(s) - lm(s - 1)) / d1 if d1 != 0 else 1.0
            x = np.zeros(1 + history * modes)
            x[0] = lm(s)
            x[1:1 + k] = a(s - 1)
            for h in range(1, history):
                x[1 + h * modes:1 + h * modes + k] = a(s - h) - a(s - h - 1)
            X.append(x)
            T.append(a(s) - a(s - 1) - rho * (a(s - 1) - a(s - 2)))
    return np.array(X), np.array(T)
