"""Device parity of the B-spline / NURBS solid bucket (FAST_ELEM_BSP_SOLID):
element matrices, assembled K and displacements against the reference's
golden dumps, and larger jittered patches against the CPU oracle.  Needs a
B200."""
import numpy as np
import pytest
import scipy.sparse as sp

from fast_b200 import decks, gpu
from oracle import fem_oracle as fo
from oracle import iga_oracle as io
from tests import golden_io as gio

pytestmark = pytest.mark.gpu

TOL_K = 1e-12
CASES = ["iga_p2_box", "iga_p3_box", "iga_scordelis_deg3"]


def loaded(name):
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    return d, g, s


@pytest.mark.parametrize("name", CASES)
def test_element_stiffness_matches_reference(name):
    d, g, s = loaded(name)
    for k, e in enumerate(g["ref_elems"]):
        Ke = s.element_matrices(int(e), 1)[0]
        assert gio.rel(Ke, g["ref_elm_K"][k]) < TOL_K, (name, e)
    s.close()


@pytest.mark.parametrize("name", CASES)
def test_assembled_matrix_matches_reference_and_is_bit_identical(name):
    d, g, s = loaded(name)
    s.assemble()
    K1 = s.lower_csr()
    R = gio.lower_K(g)
    assert K1.nnz == R.nnz
    assert abs(K1 - R).max() / abs(R).max() < TOL_K
    s.assemble()
    K2 = s.lower_csr()
    assert np.array_equal(K1.data, K2.data) and np.array_equal(K1.indices, K2.indices)
    s.close()


@pytest.mark.parametrize("prec", [gpu.PREC_FP64, gpu.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", ["iga_p2_box", "iga_p3_box"])
def test_displacements_match_reference(name, prec):
    d, g, s = loaded(name)
    s.assemble()
    f = decks.nodal_load_vector(d)
    u, rep = s.solve(f, tol=1e-12, precision=prec)
    assert rep["converged"]
    assert gio.rel(u, g["ref_u"]) < 1e-9
    s.close()


@pytest.mark.parametrize("prec", [gpu.PREC_FP64, gpu.PREC_MIXED], ids=["fp64", "mixed"])
def test_scordelis_roof_solution(prec):
    """The reference's NURBS roof (weights, degrees 3 x 3 x 2, condition number
    about 7e7) under the reference's own body-force load vector: the device
    solution agrees with the reference's skyline solution to the reference's
    own attainable accuracy (its residual is 1e-8)."""
    d, g, s = loaded("iga_scordelis_deg3")
    s.assemble()
    u, rep = s.solve(g["ref_f"], tol=1e-12, precision=prec, maxit=200000)
    assert rep["converged"]
    assert gio.rel(u, g["ref_u"]) < 2e-9
    s.close()


@pytest.mark.parametrize("p,n,rational", [(2, (6, 4, 3), True), (2, (4, 3, 3), False), (3, (4, 3, 2), True),
                                          (3, (3, 3, 3), False)])
def test_jittered_patch_matches_oracle(p, n, rational):
    """Larger patches (interior knot spans with every extraction operator
    shape) and the non-rational branch, against the Cox-de Boor oracle."""
    d = decks.bspline_box(p, n, L=(3.0, 2.0, 1.5), jitter=0.05, seed=11 + p)
    d.patch.rational = rational
    s = gpu.GpuSystem(0)
    s.upload(d)
    Kg = s.element_matrices()
    Ko = io.elems_stiff(d)
    for e in range(d.num_elems):
        assert gio.rel(Kg[e], Ko[e]) < TOL_K, e
    s.assemble()
    R = sp.tril(fo.assemble(d, Ko)).tocsr()
    K = s.lower_csr()
    assert abs(K - R).max() / abs(R).max() < TOL_K
    s.close()


def test_rejects_unsupported_patches():
    d = decks.bspline_box(2, (2, 2, 2), jitter=0.0)
    d.ngp = (2, 2, 2)  # under-integrated rule: no kernel
    s = gpu.GpuSystem(0)
    with pytest.raises(gpu.FastGpuError):
        s.upload(d)
    d = decks.bspline_box(2, (2, 2, 2), jitter=0.0)
    d.patch.span = d.patch.span.copy()
    d.patch.span[0, 0] = 7  # outside the patch
    with pytest.raises(gpu.FastGpuError):
        s.upload(d)
    s.close()


@pytest.mark.parametrize("name", ["iga_pincyl_deg4", "iga_thincyl_deg5"])
def test_high_degree_nurbs_cylinders(name):
    """The reference's own degree (4, 2, 4) and (5, 2, 5) NURBS cylinders
    (dat/iga/PinCylDeg4.dat, ThinCylinderDeg5.dat; 5- and 6-point rules): the
    layer-by-layer kernel's element matrices against the reference's dumps,
    the assembled K (bit-identical run to run) against the oracle's assembly
    of element matrices pinned to those dumps, and the solution under the
    reference's load against the reference's skyline solution."""
    d, g, s = loaded(name)
    for k, e in enumerate(g["ref_elems"]):
        Ke = s.element_matrices(int(e), 1)[0]
        assert gio.rel(Ke, g["ref_elm_K"][k]) < TOL_K, (name, e)
    s.assemble()
    K1 = s.lower_csr()
    R = sp.tril(fo.assemble(d, io.elems_stiff(d))).tocsr()
    assert K1.nnz == R.nnz
    assert abs(K1 - R).max() / abs(R).max() < TOL_K
    s.assemble()
    K2 = s.lower_csr()
    assert np.array_equal(K1.data, K2.data)
    u, rep = s.solve(g["ref_f"], tol=1e-12, precision=gpu.PREC_FP64, maxit=400000)
    assert rep["converged"]
    assert gio.rel(u, g["ref_u"]) < 1e-8
    s.close()


def test_total_lagrangian_bspline_curved_beam():
    """The reference's TL NURBS curved beam (dat/iga/CurvedBeamDeg4.dat,
    degrees 4, 2, 2, 5-point rule, load control 200 x 0.005): element
    tangents and internal forces against the reference's dumps, then the
    device Newton driver against every step the reference's `fast` binary
    printed, and the tip displacements its deck lists as expected results."""
    d, g, s = loaded("iga_curvedbeam_tl")
    n = d.num_elems
    s.set_displacement(np.zeros(d.num_eq()))
    K0 = s.element_matrices(0, n, what=gpu.ASM_K)
    for e in range(n):
        assert gio.rel(K0[e], g["ref_elm_K0"][e]) < TOL_K, e
    s.set_displacement(g["u_state"])
    Kt = s.element_matrices(0, n, what=gpu.ASM_K)
    ge = s.element_matrices(0, n, what=gpu.ASM_G)
    for e in range(n):
        assert gio.rel(Kt[e], g["ref_elm_K"][e]) < TOL_K, e
        assert gio.rel(ge[e], g["ref_elm_g"][e]) < 1e-9, e
    steps = int(g["steps"])
    hist, iters, rep = s.nr_solve(g["ref_f"], steps, float(g["step_factor"]), tol=float(g["tol"]),
                                  max_iter=int(g["maxit"]), lin_tol=1e-13)
    assert rep["converged_steps"] == steps, rep
    eq = d.node_eq()
    m = eq > 0
    tip = {}
    for k in range(steps):
        unode = np.zeros((d.num_nodes, 3))
        unode[m] = hist[k][eq[m] - 1]
        assert gio.rel(unode, g["ref_u_steps"][k]) < 1e-7, k
        tip[round(float(g["ref_lam"][k]), 6)] = unode[29]
    # "Expected displacements at the end (FAST)" in the deck's header (6 digits)
    for lf, v in ((0.30, (-5.83285, 3.49059, 28.8182)), (0.50, (-11.8457, 7.08783, 39.8952)),
                  (0.95, (-22.0535, 13.1954, 51.6480))):
        assert np.abs(tip[lf] - np.array(v)).max() <= 5e-6 * np.abs(v).max(), (lf, tip[lf])
    s.close()


@pytest.mark.parametrize("name", ["iga_p2_mass", "iga_p3_mass"])
def test_bspline_mass_matrices_match_reference(name):
    """Consistent mass of B-spline solids (cElmParam::MassMat on the
    cShapeBspSolid basis, same Gauss points as the stiffness) against the
    reference's dumps; the assembled mass is the scatter of the same blocks."""
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    for k, e in enumerate(g["ref_elems"]):
        Me = s.element_matrices(int(e), 1, what=gpu.ASM_M)[0]
        assert gio.rel(Me, g["ref_elm_M"][k]) < TOL_K, (name, e)
    s.assemble_mass()
    Ml = s.lower_csr(gpu.ASM_M)
    Ma = s.element_matrices(0, d.num_elems, what=gpu.ASM_M)
    R = sp.tril(fo.assemble(d, Ma)).tocsr()
    assert abs(Ml - R).max() / abs(R).max() < TOL_K
    s.close()
