"""Gauss-point strains and stresses on the device (fast_gpu_gauss_stress),
hex and B-spline buckets, against the reference's cElement::IntPntStress at
its own solution; nodal stresses and support reactions.  Needs a B200."""
import numpy as np
import pytest

from fast_b200 import decks, gpu
from tests import golden_io as gio

pytestmark = pytest.mark.gpu

CASES = [n for n in gio.names() if "ref_elm_stress" in gio.load(n)[1]]


@pytest.mark.parametrize("name", CASES)
def test_gauss_stress_matches_reference(name):
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.set_displacement(g["ref_u"])
    st, ss = s.gauss_stress()
    el = g["ref_elems"]
    rs, rt = g["ref_elm_stress"], g["ref_elm_strain"]
    assert np.abs(ss[el] - rs).max() <= 1e-12 * np.abs(rs).max()
    assert np.abs(st[el] - rt).max() <= 1e-12 * np.abs(rt).max()
    # a sub-range in the caller's element order
    st2, ss2 = s.gauss_stress(first=3, count=5)
    assert np.array_equal(ss2, ss[3:8])
    s.close()


def test_gauss_stress_after_device_solve():
    d, g = gio.load("cfg_hex20_lognormal_4x4x2")
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    u, rep = s.solve(g["ref_f"], tol=1e-13, precision=gpu.PREC_FP64)
    s.set_displacement(u)
    st, ss = s.gauss_stress()
    rs = g["ref_elm_stress"]
    assert np.abs(ss[g["ref_elems"]] - rs).max() <= 1e-8 * np.abs(rs).max()
    s.close()


def test_gauss_stress_rejects_total_lagrangian():
    d = decks.plate_tl_hex8(4, 4, 2)
    s = gpu.GpuSystem(0)
    s.upload(d)
    with pytest.raises(gpu.FastGpuError):
        s.gauss_stress()
    s.close()


@pytest.mark.parametrize("name", [n for n in CASES if "ref_elm_nodal_stress" in gio.load(n)[1]])
def test_nodal_stress_matches_reference_printout(name):
    """Element-nodal (cElmParam::NodalStress) and averaged nodal stresses
    (cControl::PrintAvrNodalStress) against the reference harness and the
    values the reference's `fast` binary printed to its .pos file."""
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.set_displacement(g["ref_u"])
    en, avg = s.nodal_stress()
    ref_en = g["ref_elm_nodal_stress"]
    scale = np.abs(ref_en).max()
    assert np.abs(en[g["ref_elems"]] - ref_en).max() <= 1e-12 * scale
    if "ref_pos_elm_nodal_stress" in g:
        assert np.abs(en - g["ref_pos_elm_nodal_stress"]).max() <= 1e-12 * scale
        assert np.abs(avg - g["ref_pos_nodal_stress_avg"]).max() <= 1e-12 * scale
    else:
        # (B-spline deck: no .pos printout) the average of the reference's
        # element-nodal values at each control point, in element order
        from oracle import fem_oracle as fo
        assert len(g["ref_elems"]) == d.num_elems
        ref_avg = fo.averaged_nodal_stress(d.num_nodes, d.conn, ref_en)
        assert np.abs(avg - ref_avg).max() <= 1e-12 * scale
    # run to run the same bits (gather in element order, no atomics)
    en2, avg2 = s.nodal_stress()
    assert np.array_equal(en, en2) and np.array_equal(avg, avg2)
    s.close()


def test_nodal_stress_average_on_a_mesh_with_unused_nodes():
    """Nodes of no element get zero; the averaged values are the oracle's
    arithmetic on the device's own element-nodal values."""
    from oracle import fem_oracle as fo
    d = decks.cantilever_hex8(6, 2, 2)
    extra = np.array([[50.0, 50.0, 50.0]])
    d.coords = np.vstack([d.coords, extra])
    d.fixed = np.vstack([d.fixed, [[True, True, True]]])
    s = gpu.GpuSystem(0)
    s.upload(d)
    u = np.random.default_rng(5).standard_normal(d.num_eq()) * 1e-3
    s.set_displacement(u)
    en, avg = s.nodal_stress()
    assert np.all(avg[-1] == 0.0)
    ref = fo.averaged_nodal_stress(d.num_nodes, d.conn, en)
    assert np.abs(avg - ref).max() <= 1e-14 * np.abs(ref).max()
    s.close()


@pytest.mark.parametrize("name", [n for n in CASES if "ref_reactions" in gio.load(n)[1]])
def test_support_reactions_match_reference(name):
    """fast_gpu_support_reactions (device element forces, host loads) at the
    reference's solution against the reference's cControl::SuppReactions."""
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.set_displacement(g["ref_u"])
    R = s.support_reactions()
    sup = (d.node_eq() == 0).any(axis=1)
    ref = g["ref_reactions"][:, :3]
    assert np.abs(R[sup] - ref[sup]).max() <= 1e-12 * np.abs(ref[sup]).max()
    # balance: the reactions carry the applied load
    np.testing.assert_allclose(R[sup].sum(axis=0), ref[sup].sum(axis=0), rtol=0, atol=1e-10 * np.abs(ref).max())
    s.close()


@pytest.mark.parametrize("name", ["iga_p2_box", "iga_p3_box"])
def test_bspline_nodal_stress_is_the_extrapolated_gauss_stress(name):
    """B-spline buckets: the device's element-nodal stresses are the oracle's
    extrapolation matrix (control points on the uniform natural grid) times
    the device's Gauss-point stresses, and the averages are the oracle's
    averages of them, at a seeded displacement state."""
    from oracle import fem_oracle as fo
    from oracle import iga_oracle as io
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    u = np.random.default_rng(11).standard_normal(d.num_eq()) * 1e-3
    s.set_displacement(u)
    _, ss = s.gauss_stress()
    en, avg = s.nodal_stress()
    TR = io.extrapolation_matrix(d.patch.degree, d.ngp)
    est = np.einsum("ag,egk->eak", TR, ss)
    scale = np.abs(est).max()
    assert en.shape == est.shape
    assert np.abs(en - est).max() <= 1e-13 * scale
    ref_avg = fo.averaged_nodal_stress(d.num_nodes, d.conn, en)
    assert np.abs(avg - ref_avg).max() <= 1e-14 * scale
    s.close()
