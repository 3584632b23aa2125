"""Modal analysis on the device (fast_gpu_modal) against the natural
frequencies and mode shapes the reference's own `fast` binary printed
(cCtrlModal with cGenEigSubSpaces).  Needs a B200."""
import numpy as np
import pytest

from fast_b200 import decks, gpu
from oracle import fem_oracle as fo
from tests import golden_io as gio

pytestmark = pytest.mark.gpu

CASES = ["modal_hex8_cantilever", "modal_hex20_block"]


@pytest.mark.parametrize("name", CASES)
def test_modal_matches_reference(name):
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    nm = int(g["num_modes"])
    lam, modes, rep = s.modal(nm, tol=float(g["tol"]), max_iter=int(g["maxit"]), lin_tol=1e-13)
    assert rep["converged"] == 1 and rep["subspace"] == max(2 * nm, nm + 8), rep
    # frequencies: the reference's agree with a direct sparse eigensolve to 2e-13
    assert np.abs(np.sqrt(lam) / g["ref_freq"] - 1.0).max() < 1e-10, (np.sqrt(lam), g["ref_freq"])
    # M-orthonormal modes
    M = fo.mass_matrix(d)
    G = modes @ (M @ modes.T)
    assert np.abs(G - np.eye(nm)).max() < 1e-9
    # shapes up to sign; both stopped at the reference's measure 1e-6, which
    # bounds the agreement of the vectors
    eq = d.node_eq()
    m = eq > 0
    for k in range(nm):
        node = np.zeros((d.num_nodes, 3))
        node[m] = modes[k][eq[m] - 1]
        R = g["ref_modes"][k]
        sgn = np.sign(np.sum(node * R))
        assert np.abs(sgn * node - R).max() <= 1e-5 * np.abs(R).max(), k
    # the same bits every run
    lam2, modes2, _ = s.modal(nm, tol=float(g["tol"]), max_iter=int(g["maxit"]), lin_tol=1e-13)
    assert np.array_equal(lam, lam2) and np.array_equal(modes, modes2)
    s.close()


def test_modal_reports_non_convergence():
    d, g = gio.load("modal_hex8_cantilever")
    s = gpu.GpuSystem(0)
    s.upload(d)
    with pytest.raises(gpu.FastGpuError) as ei:
        s.modal(5, tol=1e-6, max_iter=1)
    assert ei.value.rc == -5
    s.close()


def test_modal_needs_density():
    d = decks.cantilever_hex8(4, 2, 2)
    s = gpu.GpuSystem(0)
    s.upload(d)
    with pytest.raises(gpu.FastGpuError):
        s.modal(3)
    s.close()


@pytest.mark.parametrize("name", ["buck_hex8_column", "buck_hex20_column"])
def test_buckling_matches_reference(name):
    """Linear buckling (fast_gpu_buckling, cCtrlLinStab) against the
    factors and modes the reference's `fast` binary printed; the geometric
    stiffness is assembled on the device at the device's linear solution."""
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    nm = int(g["num_modes"])
    lam, modes, u, rep = s.buckling(g["ref_f"], nm, tol=float(g["tol"]), max_iter=int(g["maxit"]), lin_tol=1e-13)
    assert rep["converged"] == 1, rep
    assert gio.rel(u, g["ref_u"]) < 1e-9
    assert np.abs(lam / g["ref_lambda"] - 1.0).max() < 1e-9, (lam, g["ref_lambda"])
    eq = d.node_eq()
    m = eq > 0
    for k in range(nm):
        node = np.zeros((d.num_nodes, 3))
        node[m] = modes[k][eq[m] - 1]
        R = g["ref_modes"][k]
        sgn = np.sign(np.sum(node * R))
        assert np.abs(sgn * node - R).max() <= 1e-5 * np.abs(R).max(), k
    s.close()
