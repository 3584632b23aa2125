"""Generalized eigenproblem K v = lambda M v by subspace iteration on the CPU
(TEST INFRASTRUCTURE ONLY).

A restatement of cGenEigSubSpaces::Solver (mlib/eig.cpp:377-510) as
cCtrlModal::Solver (ctrl/ctrlmodal.cpp:48-128) drives it:

  q = max(2 p, p + 8) vectors; start: unit vectors at the q smallest
  K_ii / M_ii (ties by equation), the last one an alternating-sign random
  vector; each iteration  K Y = M X  (X itself at the first), the projected
  Kp = Y^T K Y, Mp = Y^T M Y, their eigenpairs Kp phi = lambda Mp phi with
  phi^T Mp phi = 1 ascending, X = Y Phi; converged when every one of the p
  lowest has sqrt(|1 - lambda^2 / |phi|^2|) <= tol.

cCtrlLinStab::Solver (ctrl/ctrllinstab.cpp:46-140) runs the same iteration
on K v = lambda (-G) v, G the geometric stiffness at the linear solution of
the reference load (cControl::GeomStiffMatrix); lambda are the buckling
factors.

Here the K solves are sparse LU and the projected problem is solved by a
Cholesky reduction and a symmetric eigensolver instead of the reference's
generalized Jacobi sweeps (cGenEigJacobi, mlib/eig.cpp:528-722): the same
eigenpairs and normalisation, up to the sign of each vector.  Frequencies
are sqrt(lambda) (cCtrlModal::Solver).

Only ``tests/`` imports this module.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sl
import scipy.sparse.linalg as sla


def start_vectors(K, M, q, seed=1):
    """[q][n] starting vectors of cGenEigSubSpaces::Solver."""
    n = K.shape[0]
    kd, md = K.diagonal(), M.diagonal()
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(md != 0.0, kd / np.where(md != 0.0, md, 1.0), np.inf)
    order = sorted(range(n), key=lambda i: (ratio[i], i))
    X = np.zeros((q, n))
    for j in range(q):
        X[j, order[j]] = 1.0
    rng = np.random.default_rng(seed)
    last = rng.random(n) * np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    X[q - 1] = last / np.linalg.norm(last)
    return X


def projected_eigen(Kp, Mp):
    """Eigenpairs of Kp phi = lambda Mp phi, ascending, phi^T Mp phi = 1."""
    lam, Phi = sl.eigh(0.5 * (Kp + Kp.T), 0.5 * (Mp + Mp.T))
    return lam, Phi


def projected_eigen_swapped(Kp, Bp):
    """The same pencil when Bp need not be definite (buckling, Bp = -Y^T G Y):
    Bp z = mu Kp z with z^T Kp z = 1, lambda = 1 / mu, phi = z / sqrt(|mu|),
    ascending in lambda as sEigPair::ComparePair orders them."""
    mu, Z = sl.eigh(0.5 * (Bp + Bp.T), 0.5 * (Kp + Kp.T))
    with np.errstate(divide="ignore"):
        lam = np.where(mu != 0.0, 1.0 / mu, np.inf)
    Phi = Z / np.sqrt(np.where(mu != 0.0, np.abs(mu), 1.0))
    order = np.argsort(lam, kind="stable")
    return lam[order], Phi[:, order]


def subspace(K, M, p, tol, maxit, X0=None, swapped=False):
    """(lambda [p], modes [p][n] with v^T M v = 1, iterations, converged).
    M is the right-hand matrix of the pencil: the mass for modal analysis,
    minus the geometric stiffness for linear buckling (swapped=True)."""
    n = K.shape[0]
    q = min(max(2 * p, p + 8), n)
    X = start_vectors(K, M, q) if X0 is None else X0
    lu = sla.splu(K.tocsc())
    lam = None
    for it in range(maxit):
        Y = np.array([lu.solve(X[i] if it == 0 else M @ X[i]) for i in range(q)])
        Kp = Y @ (K @ Y.T)
        Mp = Y @ (M @ Y.T)
        lam, Phi = projected_eigen_swapped(Kp, Mp) if swapped else projected_eigen(Kp, Mp)
        X = (Y.T @ Phi).T
        err = np.sqrt(np.abs(1.0 - lam[:p] ** 2 / np.sum(Phi[:, :p] ** 2, axis=0)))
        if np.all(err <= tol):
            return lam[:p], X[:p], it + 1, True
    return lam[:p], X[:p], maxit, False
