"""Pin the B-spline / NURBS solid oracle (oracle/iga_oracle.py) against golden
vectors dumped from the reference FAST program, and check the deck side of
%PATCH / %ELEMENT.BSPLINE.SOLID.  CPU only."""
import numpy as np
import pytest
import scipy.sparse as sp

from fast_b200 import decks
from oracle import fem_oracle as fo
from oracle import iga_oracle as io
from tests import golden_io as gio

CASES = ["iga_p2_box", "iga_p3_box", "iga_scordelis_deg3", "iga_pincyl_deg4", "iga_thincyl_deg5"]


@pytest.mark.parametrize("name", CASES)
def test_equation_numbering(name):
    d, g = gio.load(name)
    assert d.num_eq() == int(g["ref_neq"][0])
    np.testing.assert_array_equal(d.node_eq(), g["ref_node_eq"])
    np.testing.assert_array_equal(fo.elem_dofs(d), g["ref_elm_dofs"])


@pytest.mark.parametrize("name", CASES)
def test_element_stiffness(name):
    d, g = gio.load(name)
    el = g["ref_elems"]
    Ke = io.elems_stiff(d, el)
    for k in range(len(el)):
        assert gio.rel(Ke[k], g["ref_elm_K"][k]) < 1e-13, (name, k)


@pytest.mark.parametrize("name", ["iga_p2_box", "iga_p3_box"])
def test_assembled_matrix_load_and_displacements(name):
    d, g = gio.load(name)
    K = fo.assemble(d, io.elems_stiff(d))
    R = gio.lower_K(g)
    Kl = sp.tril(K).tocsr()
    assert abs(Kl - R).max() / abs(R).max() < 1e-13
    assert Kl.nnz == R.nnz
    f = decks.nodal_load_vector(d)
    assert gio.rel(f, g["ref_f"]) < 1e-15
    u, ok, it, err = fo.pcg(K, f, 1e-13, 100000)
    assert ok
    assert gio.rel(u, g["ref_u"]) < 1e-9


def test_scordelis_matrix_and_reference_solution():
    """NURBS deck with weights: assembled K from the oracle's element matrices
    equals the reference's, and K u = f with the reference's load gives its u."""
    d, g = gio.load("iga_scordelis_deg3")
    assert d.patch.rational and d.patch.weights is not None
    assert d.patch.degree == (3, 3, 2)
    K = fo.assemble(d, io.elems_stiff(d))
    R = gio.lower_K(g)
    assert abs(sp.tril(K).tocsr() - R).max() / abs(R).max() < 1e-13
    r = g["ref_f"] - K @ g["ref_u"]
    assert np.linalg.norm(r) / np.linalg.norm(g["ref_f"]) < 1e-8


def test_written_deck_reads_back(tmp_path):
    d = decks.bspline_box(3, (3, 2, 2), jitter=0.05, seed=4)
    base = str(tmp_path / "b")
    decks.write_dat(d, base)
    r = decks.read_dat(base + ".dat")
    assert r.kind == "bsp" and r.patch.degree == (3, 3, 3) and r.ngp == (4, 4, 4)
    np.testing.assert_array_equal(r.conn, d.conn)
    np.testing.assert_allclose(r.coords, d.coords, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(r.patch.span, d.patch.span)
    for k in range(3):
        np.testing.assert_array_equal(r.patch.knots[k], d.patch.knots[k])


def test_unit_weight_nurbs_equals_bspline():
    """With unit weights the rational quotient is the plain tensor product."""
    d = decks.bspline_box(2, (2, 2, 2), jitter=0.05, seed=5)
    Kr = io.elem_stiff(d, 3)
    d.patch.rational = False
    Kp = io.elem_stiff(d, 3)
    assert gio.rel(Kp, Kr) < 1e-13


@pytest.mark.parametrize("name", ["iga_pincyl_deg4", "iga_thincyl_deg5"])
def test_high_degree_cylinders_solution(name):
    """dat/iga/PinCylDeg4.dat and ThinCylinderDeg5.dat: K assembled from the
    oracle's element matrices solves the reference's load to the reference's
    skyline solution."""
    import scipy.sparse.linalg as sla
    d, g = gio.load(name)
    assert d.patch.rational and d.patch.degree in ((4, 2, 4), (5, 2, 5))
    K = fo.assemble(d, io.elems_stiff(d))
    u = sla.spsolve(K.tocsc(), g["ref_f"])
    assert gio.rel(u, g["ref_u"]) < 1e-8


def test_total_lagrangian_bspline_element():
    """dat/iga/CurvedBeamDeg4.dat (%ELEMENT.BSPLINE.SOLIDTL, degrees 4, 2, 2):
    the oracle's TL tangent at u = 0 and the TL tangent and internal force at
    a state of the reference's own load path, against the harness dumps."""
    d, g = gio.load("iga_curvedbeam_tl")
    assert d.total_lagrangian and d.patch.degree == (4, 2, 2)
    np.testing.assert_array_equal(d.node_eq(), g["ref_node_eq"])
    eq = d.node_eq()
    m = eq > 0
    unode = np.zeros((d.num_nodes, 3))
    unode[m] = g["u_state"][eq[m] - 1]
    for e in range(d.num_elems):
        K0, _ = io.elem_tl(d, e, np.zeros(3 * d.nn))
        assert gio.rel(K0, g["ref_elm_K0"][e]) < 1e-13
        Kt, ge = io.elem_tl(d, e, unode[d.conn[e]].ravel())
        assert gio.rel(Kt, g["ref_elm_K"][e]) < 1e-13
        # the force at a large-rotation, small-strain state loses digits to
        # cancellation in F^T F - I
        assert gio.rel(ge, g["ref_elm_g"][e]) < 1e-9


def test_bspline_gauss_point_stresses():
    """cElement::IntPntStress of a B-spline solid at the reference's solution
    (strains and stresses of every Gauss point) from the oracle."""
    d, g = gio.load("iga_p2_box")
    eq = d.node_eq()
    m = eq > 0
    un = np.zeros((d.num_nodes, 3))
    un[m] = g["ref_u"][eq[m] - 1]
    for k, e in enumerate(g["ref_elems"]):
        st, ss = io.elem_stress(d, int(e), un[d.conn[e]].ravel())
        assert np.abs(st - g["ref_elm_strain"][k]).max() <= 1e-12 * np.abs(g["ref_elm_strain"]).max()
        assert np.abs(ss - g["ref_elm_stress"][k]).max() <= 1e-12 * np.abs(g["ref_elm_stress"]).max()


def test_bspline_extrapolation_matches_reference_nodal_stress():
    """The restated CompTRMatrix for a B-spline element (least squares through
    the Gauss points, evaluated on the control points' uniform natural grid)
    times the reference's Gauss-point stresses gives the element-nodal
    stresses the reference's cElmParam::NodalStress returned."""
    d, g = gio.load("iga_p2_box")
    TR = io.extrapolation_matrix(d.patch.degree, d.ngp)
    est = np.einsum("ag,egk->eak", TR, g["ref_elm_stress"])
    ref = g["ref_elm_nodal_stress"]
    assert np.abs(est - ref).max() <= 1e-12 * np.abs(ref).max()
