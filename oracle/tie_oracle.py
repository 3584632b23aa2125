"""Multi-block assembly and tied-interface elimination on the CPU (TEST
INFRASTRUCTURE ONLY).

The tie  u_s = sum_k w_k u_(m_k)  (x, y, z) is the reference's linear
multi-point constraint (%NODE.MULTI-POINT.CONSTRAINT, node/node.cpp:459-509).
The reference enforces it with Lagrange multipliers (cSysMatrix::SolveMPC,
mlib/sysmat.cpp:72-143: K B = P^T, A = P B, solve for the multipliers); for a
homogeneous constraint set whose slave DOFs appear in no other constraint that
has the same solution as eliminating the slaves, u = T u~, which this module
does with scipy in equation space:

    K~ = T^T K T,  f~ = T^T f,  K~_rr u~_r = f~_r,  u = T u~ .

Element matrices come from the other checkers: hex8 / hex20 from the C
restatement (fem_oracle), B-spline solids from iga_oracle.  Only ``tests/``
imports this module.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import fem_oracle as fo
from . import iga_oracle as io


def bucket_matrices(deck, b):
    return io.elems_stiff(b) if b.kind == "bsp" else fo.elems_stiff(b)[0]


def assemble(deck):
    """Equation-space K of all buckets of a multi-block deck (caller numbering)."""
    eq = deck.node_eq()
    neq = int(eq.max(initial=0))
    I, J, V = [], [], []
    for b in deck.buckets():
        Ke = bucket_matrices(deck, b)
        dofs = eq[b.conn].reshape(b.num_elems, -1)
        nd = dofs.shape[1]
        Ii = np.repeat(dofs, nd, axis=1).ravel()
        Jj = np.tile(dofs, (1, nd)).ravel()
        Vv = Ke.reshape(len(dofs), -1).ravel()
        m = (Ii > 0) & (Jj > 0)
        I.append(Ii[m] - 1); J.append(Jj[m] - 1); V.append(Vv[m])
    K = sp.csr_matrix((np.concatenate(V), (np.concatenate(I), np.concatenate(J))), shape=(neq, neq))
    K.sum_duplicates()
    K.sort_indices()
    return K


def tie_matrix(deck):
    """T (equation space): identity on non-slave equations; slave equation
    (s, i) maps to the masters' equations (m_k, i) with weight w_k."""
    eq = deck.node_eq()
    neq = int(eq.max(initial=0))
    t = deck.ties
    slave_eq = np.zeros(neq, bool)
    rows, cols, vals = [], [], []
    for k, s in enumerate(t.slave):
        for i in range(3):
            es = eq[s, i]
            if es == 0:
                continue
            slave_eq[es - 1] = True
            for q in range(t.ptr[k], t.ptr[k + 1]):
                em = eq[t.master[q], i]
                if em:
                    rows.append(es - 1); cols.append(em - 1); vals.append(t.weight[q])
    keep = np.nonzero(~slave_eq)[0]
    rows += list(keep); cols += list(keep); vals += [1.0] * len(keep)
    T = sp.csr_matrix((vals, (rows, cols)), shape=(neq, neq))
    return T, slave_eq


def reduced(deck, K=None):
    """(K~ with unit diagonal on the slave equations, T, slave mask)."""
    if K is None:
        K = assemble(deck)
    T, slave = tie_matrix(deck)
    Kt = (T.T @ K @ T).tocsr()
    Kt = Kt + sp.diags(slave.astype(np.float64))
    Kt.sum_duplicates()
    Kt.sort_indices()
    return Kt.tocsr(), T, slave


def solve(deck, f, tol=1e-13, maxit=200000, K=None):
    """u = T u~ with K~ u~ = T^T f solved by the reference's Jacobi PCG."""
    Kt, T, slave = reduced(deck, K)
    ft = T.T @ f
    ft[slave] = 0.0
    ut, ok, it, err = fo.pcg(Kt, ft, tol, maxit)
    return T @ ut, ok, it


def solve_full(deck, tol=1e-13, maxit=500000):
    """solve() for the full-size column: nodal load of the deck, the PCG on all
    host threads; returns u and a dict of what the fixture records."""
    from fast_b200 import decks
    f = decks.nodal_load_vector(deck)
    K = assemble(deck)
    Kt, T, slave = reduced(deck, K)
    ft = T.T @ f
    ft[slave] = 0.0
    ut, it, err = fo.pcg_threaded(Kt, ft, tol, maxit)
    u = T @ ut
    true_res = np.linalg.norm(ft - Kt @ ut) / np.linalg.norm(ft)
    return u, dict(iterations=it, rec_err=err, true_rel_residual=true_res, neq=K.shape[0],
                   f_norm2=np.linalg.norm(f), nnz_reduced=Kt.nnz)
