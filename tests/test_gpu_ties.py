"""Device parity of tied interfaces (slave DOFs eliminated, K~ = T^T K T
assembled directly): the reduced matrix, its run-to-run bit identity and the
displacements against the CPU elimination oracle, on a four-block column
(B-spline p=2, hex8, hex20, B-spline p=3) with non-matching interfaces.
Needs a B200."""
import numpy as np
import pytest
import scipy.sparse as sp

from fast_b200 import decks, gpu
from oracle import tie_oracle as to
from tests import golden_io as gio

pytestmark = pytest.mark.gpu


def column():
    return decks.tied_column(hex8=(4, 4, 2), hex20=(3, 3, 2), p2=(3, 3, 2), p3=(2, 2, 2), jitter=0.05, seed=3)


def test_reduced_matrix_matches_oracle_and_is_bit_identical():
    d = column()
    Kt, T, slave = to.reduced(d)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    K1 = s.lower_csr()
    R = sp.tril(Kt).tocsr()
    D = (K1 - R).tocsr()
    D.eliminate_zeros()
    assert D.nnz == 0 or abs(D).max() / abs(R).max() < 1e-12
    s.assemble()
    K2 = s.lower_csr()
    assert np.array_equal(K1.data, K2.data) and np.array_equal(K1.indices, K2.indices)
    s.close()


@pytest.mark.parametrize("prec", [gpu.PREC_FP64, gpu.PREC_MIXED], ids=["fp64", "mixed"])
def test_tied_displacements_match_oracle(prec):
    d = column()
    f = decks.nodal_load_vector(d)
    u_o, ok, it = to.solve(d, f)
    assert ok
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    u, rep = s.solve(f, tol=1e-12, precision=prec)
    assert rep["converged"]
    assert gio.rel(u, u_o) < 1e-9
    # the slaves sit on their master surfaces
    eq = d.node_eq()
    t = d.ties
    for k in range(0, len(t.slave), 7):
        sl = t.slave[k]
        ms, ws = t.master[t.ptr[k]:t.ptr[k + 1]], t.weight[t.ptr[k]:t.ptr[k + 1]]
        for i in range(3):
            if eq[sl, i]:
                um = np.array([u[eq[m, i] - 1] if eq[m, i] else 0.0 for m in ms])
                assert abs(u[eq[sl, i] - 1] - ws @ um) <= 1e-12 * np.abs(u).max()
    s.close()


def test_ties_reject_other_analyses():
    d = column()
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    with pytest.raises(gpu.FastGpuError):
        s.internal_force()
    s.close()
