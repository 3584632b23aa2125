"""Tied interfaces on the host: tie weights reproduce the slave positions,
the host pattern covers T^T K T, and the CPU elimination agrees with the
reference's Lagrange-multiplier form of the same constraints.  CPU only."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from fast_b200 import decks, gpu
from oracle import tie_oracle as to


def small():
    return decks.tied_column(hex8=(4, 4, 2), hex20=(3, 3, 2), p2=(3, 3, 2), p3=(2, 2, 2), jitter=0.05, seed=3)


def test_tie_weights_interpolate_the_slave_positions():
    d = small()
    t = d.ties
    assert len(t.slave) == 5 * 5 * 2 + (7 * 7 - 9)  # hex8 bottom and top faces, hex20 top face
    for k, s in enumerate(t.slave):
        ms, ws = t.master[t.ptr[k]:t.ptr[k + 1]], t.weight[t.ptr[k]:t.ptr[k + 1]]
        assert abs(ws.sum() - 1.0) < 1e-13
        np.testing.assert_allclose(ws @ d.coords[ms], d.coords[s], rtol=0, atol=1e-13)
    assert not set(t.slave) & set(t.master)


def test_host_pattern_covers_the_reduced_matrix():
    d = small()
    p = gpu.inspect_pattern(d)
    Kt, T, slave = to.reduced(d)
    eq = d.node_eq()
    rp, col = p["rowptr"], p["col"]
    blocks = set()
    for n in range(d.num_nodes):
        for c in col[rp[n]:rp[n + 1]]:
            blocks.add((n, int(c)))
    node_of = np.zeros(Kt.shape[0], np.int64)
    for n in range(d.num_nodes):
        for i in range(3):
            if eq[n, i]:
                node_of[eq[n, i] - 1] = n
    C = Kt.tocoo()
    for i, j in zip(C.row, C.col):
        assert (node_of[i], node_of[j]) in blocks


def test_elimination_equals_lagrange_multipliers():
    """[K P^T; P 0] [u; lambda] = [f; 0] (the reference's SolveMPC system) has
    the same displacements as the eliminated solve."""
    d = small()
    K = to.assemble(d)
    f = decks.nodal_load_vector(d)
    u_e, ok, it = to.solve(d, f, K=K)
    assert ok
    T, slave = to.tie_matrix(d)
    # constraint rows: u_s - T_s u = 0 for every slave equation
    P = (sp.identity(K.shape[0], format="csr") - T)[np.nonzero(slave)[0]]
    A = sp.bmat([[K, P.T], [P, None]]).tocsc()
    x = spla.spsolve(A, np.concatenate([f, np.zeros(P.shape[0])]))
    u_l = x[:K.shape[0]]
    assert np.abs(u_e - u_l).max() / np.abs(u_l).max() < 1e-9
