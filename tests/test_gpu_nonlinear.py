"""Device parity of the total-Lagrangian element, the internal force and the
load-control Newton driver (through the C ABI) against the reference."""
import numpy as np
import pytest
import scipy.sparse as sp

from fast_b200 import decks, gpu
from oracle import fem_oracle as fo
from tests import golden_io as gio

pytestmark = pytest.mark.gpu

TOL_K = 1e-12


def system(d):
    s = gpu.GpuSystem(0)
    s.upload(d)
    return s


def _assemble_vec(d, elm_vals):
    dofs = fo.elem_dofs(d)
    g = np.zeros(d.num_eq())
    for e in range(d.num_elems):
        m = dofs[e] > 0
        np.add.at(g, dofs[e][m] - 1, elm_vals[e][m])
    return g


def test_tl_element_tangent_and_force_match_reference():
    d, g = gio.load("cfg_hex8_tl_state")
    s = system(d)
    s.set_displacement(g["u_state"])
    Kt = s.element_matrices(0, d.num_elems, what=gpu.ASM_K)
    ge = s.element_matrices(0, d.num_elems, what=gpu.ASM_G)
    for k, e in enumerate(g["ref_elems"]):
        assert gio.rel(Kt[e], g["ref_elm_K"][k]) < TOL_K, e
        assert gio.rel(ge[e], g["ref_elm_g"][k]) < 1e-12, e
    # assembled internal force and tangent
    gg = s.internal_force()
    assert gio.rel(gg, _assemble_vec(d, g["ref_elm_g"])) < 1e-12
    s.assemble()
    Kl = s.lower_csr()
    R = sp.tril(fo.assemble(d, g["ref_elm_K"])).tocsr()
    assert abs(Kl - R).max() / abs(R).max() < TOL_K


def test_small_strain_internal_force_matches_reference():
    d, g = gio.load("cfg_hex20_lognormal_4x4x2")
    s = system(d)
    s.set_displacement(g["ref_u"])
    assert gio.rel(s.internal_force(), g["ref_g_of_u"]) < 1e-10


@pytest.mark.parametrize("precision", [gpu.PREC_FP64, gpu.PREC_MIXED])
@pytest.mark.parametrize("predictor", [gpu.PREDICT_NONE, gpu.PREDICT_SECANT])
def test_newton_matches_reference_cctrlnr(precision, predictor):
    """Every load step of the device Newton equals the displacements the
    reference's own cCtrlNR printed (TL hex8 plate, 4 steps)."""
    d, g = gio.load("nr_plate_tl")
    s = system(d)
    hist, iters, rep = s.nr_solve(g["ref_f"], int(g["steps"]), float(g["step_factor"]), tol=float(g["tol"]),
                                  max_iter=int(g["maxit"]), predictor=predictor, precision=precision,
                                  lin_tol=1e-12)
    assert rep["converged_steps"] == int(g["steps"]) and (iters > 0).all()
    eq = d.node_eq()
    m = eq > 0
    for k in range(hist.shape[0]):
        unode = np.zeros((d.num_nodes, 3))
        unode[m] = hist[k][eq[m] - 1]
        assert gio.rel(unode, g["ref_u_steps"][k]) < 1e-8, (k, iters, rep)


def test_secant_predictor_saves_newton_iterations():
    d = decks.plate_tl_hex8(10, 10, 2, L=4.0, t=0.4, pressure=12.0, steps=8, tol=1e-8)
    s = system(d)
    q = gpu.face_load_vector(d)
    h0, it0, r0 = s.nr_solve(q, 8, 1 / 8, tol=1e-8, predictor=gpu.PREDICT_NONE, precision=gpu.PREC_MIXED,
                             lin_tol_rel=1e-3)
    h1, it1, r1 = s.nr_solve(q, 8, 1 / 8, tol=1e-8, predictor=gpu.PREDICT_SECANT, precision=gpu.PREC_MIXED,
                             lin_tol_rel=1e-3)
    assert r0["converged_steps"] == 8 and r1["converged_steps"] == 8
    assert r1["iterations"] < r0["iterations"], (it0, it1)
    assert gio.rel(h1[-1], h0[-1]) < 1e-6


def test_newton_reports_failure():
    d = decks.plate_tl_hex8(4, 4, 2, L=4.0, t=0.4, pressure=8.0, steps=2, tol=1e-14)
    s = system(d)
    q = gpu.face_load_vector(d)
    with pytest.raises(gpu.FastGpuError) as ei:
        s.nr_solve(q, 2, 0.5, tol=1e-30, max_iter=3)
    assert ei.value.rc == -5


@pytest.mark.parametrize("method", ["ioal", "uoal", "clinal"])
def test_arclength_matches_reference_cctrlpath(method):
    """Every step of the device arc-length driver equals the displacements and
    load factors the reference's own cCtrlPath printed (TL hex8 plate, 8
    steps, TargetIter 4)."""
    d, g = gio.load("arc_plate_tl")
    s = system(d)
    hist, lams, iters, rep = s.arclength_solve(g["ref_f"], method, int(g["steps"]), float(g["step_factor"]),
                                               tol=float(g["tol"]), max_iter=int(g["maxit"]),
                                               load_coeff=float(g["load_coeff"]), target_iter=int(g["target_iter"]))
    ref_lam = g["ref_lam_" + method]
    assert rep["converged_steps"] == len(ref_lam), rep
    assert np.abs(lams - ref_lam).max() < 1e-9, (lams, ref_lam)
    eq = d.node_eq()
    m = eq > 0
    for k in range(hist.shape[0]):
        unode = np.zeros((d.num_nodes, 3))
        unode[m] = hist[k][eq[m] - 1]
        assert gio.rel(unode, g["ref_u_steps_" + method][k]) < 1e-8, (k, iters, rep)


def test_arclength_reports_failure():
    d = decks.plate_tl_hex8(4, 4, 2, L=4.0, t=0.4, pressure=8.0, steps=2, tol=1e-14)
    s = system(d)
    q = gpu.face_load_vector(d)
    with pytest.raises(gpu.FastGpuError) as ei:
        s.arclength_solve(q, "clinal", 2, 0.5, tol=1e-30, max_iter=3)
    assert ei.value.rc == -5


@pytest.mark.parametrize("precision", [gpu.PREC_FP64, gpu.PREC_MIXED])
def test_newton_graph_replay_equals_direct_launches(precision):
    """Newton iterations after the first replay one captured CUDA graph
    (tangent, preconditioner, the PCG as a conditional WHILE node, update,
    internal force, norms); kernel-by-kernel launches give the same steps."""
    d = decks.plate_tl_hex8(8, 8, 2, L=4.0, t=0.4, pressure=10.0, steps=6, tol=1e-8)
    q = gpu.face_load_vector(d)
    s = system(d)
    kw = dict(tol=1e-8, predictor=gpu.PREDICT_SECANT, precision=precision, lin_tol=1e-10,
              lin_tol_rel=1e-3 if precision == gpu.PREC_MIXED else 0.0)
    h1, it1, r1 = s.nr_solve(q, 6, 1 / 6, **kw)
    s.set_option(gpu.OPT_GRAPH_STEPS, 0)
    h0, it0, r0 = s.nr_solve(q, 6, 1 / 6, **kw)
    assert r1["converged_steps"] == r0["converged_steps"] == 6
    if precision == gpu.PREC_FP64:
        # the same iteration, so the same Newton iterations
        assert (it1 == it0).all(), (it1, it0)
        assert gio.rel(h1, h0) < 1e-10
    else:
        # the FP32 iteration runs in other kernels (the replayed loop's
        # persistent chunks against the direct solves): both meet the Newton
        # tolerance
        assert gio.rel(h1, h0) < 1e-7
    s.close()


@pytest.mark.parametrize("which", ["tl_plate", "hex20_box", "two_buckets"])
def test_gathered_internal_force_equals_colour_scatter(which):
    """FAST_OPT_FORCE_GATHER: the internal force formed element by element in
    one launch per bucket and gathered per node (in bucket, then colour order)
    is the same bits as the colour-by-colour scatter, in fewer launches; so
    are the Newton steps built on it."""
    import dataclasses
    if which == "tl_plate":
        d = decks.plate_tl_hex8(8, 8, 2, L=4.0, t=0.4, pressure=10.0, steps=6, tol=1e-8)
    elif which == "hex20_box":
        d = decks.box_hex20_lognormal(6, 6, 3, seed=9)
    else:
        # two hex20 buckets sharing their interface nodes (3x3x3 and 2x2x2 rules)
        d0 = decks.box_hex20_lognormal(6, 6, 4, seed=6)
        h = d0.num_elems // 2
        nofaces = dict(face_elem=None, face_corners=None, face_q=None, face_local=None, blocks=[])
        blk = dataclasses.replace(d0, conn=d0.conn[h:], E=d0.E[h:], nu=d0.nu[h:], ngp=(2, 2, 2), **nofaces)
        d = dataclasses.replace(d0, conn=d0.conn[:h], E=d0.E[:h], nu=d0.nu[:h], **nofaces)
        d.blocks = [blk]
    s = system(d)
    u = np.random.default_rng(5).standard_normal(d.num_eq()) * 1e-2
    s.set_displacement(u)
    g = {}
    launches = {}
    for opt in (1, 0):
        s.set_option(gpu.OPT_FORCE_GATHER, opt)
        n0 = s.launch_count()
        g[opt] = s.internal_force()
        launches[opt] = s.launch_count() - n0
    assert np.array_equal(g[1], g[0]) and np.abs(g[0]).max() > 0
    assert launches[1] <= launches[0], launches
    if which == "tl_plate":
        q = gpu.face_load_vector(d)
        kw = dict(tol=1e-8, predictor=gpu.PREDICT_SECANT, precision=gpu.PREC_FP64, lin_tol=1e-10)
        h = {}
        for opt in (1, 0):
            s.set_option(gpu.OPT_FORCE_GATHER, opt)
            h[opt], _, r = s.nr_solve(q, 6, 1 / 6, **kw)
            assert r["converged_steps"] == 6
        assert np.array_equal(h[1], h[0])
    s.close()
