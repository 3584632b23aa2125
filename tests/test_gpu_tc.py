"""The tensor-core stiffness (FAST_ASM_STIFFNESS_TF32: element products on
tcgen05 in 3xTF32, FP32 blocks) and the mixed-precision solve on it, whose
FP64 residuals are formed element by element.

Bounds: the element matrices agree with the reference's StiffMat dumps to
TOL_TF32 relative to the largest entry (3xTF32 keeps about 21 bits per
product; FP32 accumulation over the Gauss points), and the displacements
after the FP64 refinement meet the same 1e-9 as the FP64 path."""
import numpy as np
import pytest
import scipy.sparse as sp

from fast_b200 import decks, gpu
from oracle import fem_oracle as fo
from tests import golden_io as gio

pytestmark = pytest.mark.gpu

TOL_TF32 = 2e-6
TOL_U = 1e-9


def system(d):
    s = gpu.GpuSystem(0)
    s.upload(d)
    return s


@pytest.mark.parametrize("name", ["cfg_hex8_cantilever", "cfg_hex20_lognormal_4x4x2"])
def test_tensor_core_element_matrices_match_reference(name):
    d, g = gio.load(name)
    s = system(d)
    worst = 0.0
    for k, e in enumerate(g["ref_elems"]):
        Ke = s.element_matrices(int(e), 1, what=gpu.ASM_K_TF32)[0]
        err = gio.rel(Ke, g["ref_elm_K"][k])
        worst = max(worst, err)
        assert err < TOL_TF32, (e, err)
        assert np.abs(Ke - Ke.T).max() <= 1e-12 * np.abs(Ke).max()
    print(name, "worst element error vs the reference %.2e" % worst)
    s.close()


def test_tensor_core_stiffness_is_deterministic_and_close_to_fp64():
    d = decks.box_hex20_lognormal(8, 8, 4, seed=3)
    s = system(d)
    s.assemble()
    K64 = s.lower_csr()
    s.assemble(gpu.ASM_K_TF32)
    K1 = s.lower_csr(gpu.ASM_K_TF32)
    s.assemble(gpu.ASM_K_TF32)
    K2 = s.lower_csr(gpu.ASM_K_TF32)
    assert (K1 != K2).nnz == 0  # bit-identical run to run
    assert abs(K1 - K64).max() / abs(K64).max() < TOL_TF32
    s.close()


# solver tolerance per deck: the slender cantilever's attainable FP64
# residual is about 1e-11 (the reference's own skyline solution has 4.7e-11)
SOLVE_TOL = {"cfg_hex8_cantilever": 1e-10}


@pytest.mark.parametrize("name", ["cfg_hex8_cantilever", "cfg_hex20_lognormal_4x4x2"])
def test_mixed_solve_on_tensor_core_stiffness_matches_reference(name):
    d, g = gio.load(name)
    s = system(d)
    s.assemble(gpu.ASM_K_TF32)
    tol = SOLVE_TOL.get(name, 1e-12)
    u, rep = s.solve(g["ref_f"], tol=tol, precision=gpu.PREC_MIXED)
    assert rep["converged"] and rep["true_rel_residual"] < tol, rep
    assert gio.rel(u, g["ref_u"]) < TOL_U, (rep, gio.rel(u, g["ref_u"]))
    # an FP64 solve needs the FP64 stiffness
    with pytest.raises(gpu.FastGpuError) as ei:
        s.solve(g["ref_f"], tol=1e-12, precision=gpu.PREC_FP64)
    assert ei.value.rc == -4
    s.assemble()
    u64, rep64 = s.solve(g["ref_f"], tol=1e-12, precision=gpu.PREC_FP64)
    assert gio.rel(u, u64) < TOL_U
    s.close()


def test_tensor_core_path_on_medium_hex20_box_against_oracle():
    d = decks.box_hex20_lognormal(16, 16, 8, seed=2)
    s = system(d)
    s.assemble(gpu.ASM_K_TF32)
    f = gpu.face_load_vector(d)
    K = fo.assemble(d)
    u_o, ok, it, err = fo.pcg(K, f, 1e-12, 100000)
    assert ok
    for tol in (1e-8, 1e-10):
        u, rep = s.solve(f, tol=tol, precision=gpu.PREC_MIXED)
        assert rep["converged"], rep
        tr = np.linalg.norm(f - K @ u) / np.linalg.norm(f)
        assert tr < tol, (tol, tr, rep)
        print("tol %.0e: %d iterations, %d FP64 residuals, |u - u_oracle|/|u_oracle| %.2e"
              % (tol, rep["iterations"], rep["outer"], gio.rel(u, u_o)))
    assert gio.rel(u, u_o) < TOL_U
    s.close()


def test_tensor_core_stiffness_rejects_total_lagrangian_buckets():
    d = decks.plate_tl_hex8(4, 4, 2, L=4.0, t=0.4, pressure=8.0, steps=2)
    s = system(d)
    with pytest.raises(gpu.FastGpuError) as ei:
        s.assemble(gpu.ASM_K_TF32)
    assert ei.value.rc == -7
    s.close()


@pytest.mark.parametrize("name", ["iga_p2_box", "iga_p3_box", "iga_scordelis_deg3"])
def test_bspline_tensor_core_element_matrices_match_reference(name):
    """B-spline solids (degrees (2,2,2), (3,3,3) and the NURBS roof's (3,3,2),
    whose left-handed parametrisation gives negative Gauss weights c_g)."""
    d, g = gio.load(name)
    s = system(d)
    worst = 0.0
    for k, e in enumerate(g["ref_elems"]):
        Ke = s.element_matrices(int(e), 1, what=gpu.ASM_K_TF32)[0]
        err = gio.rel(Ke, g["ref_elm_K"][k])
        worst = max(worst, err)
        assert err < TOL_TF32, (e, err)
        assert np.abs(Ke - Ke.T).max() == 0.0   # symmetric by construction
    print(name, "worst element error vs the reference %.2e" % worst)
    s.close()


@pytest.mark.parametrize("name", ["iga_p2_box", "iga_p3_box"])
def test_bspline_mixed_solve_on_tensor_core_stiffness(name):
    d, g = gio.load(name)
    s = system(d)
    s.assemble(gpu.ASM_K_TF32)
    K1 = s.lower_csr(gpu.ASM_K_TF32)
    s.assemble(gpu.ASM_K_TF32)
    assert (s.lower_csr(gpu.ASM_K_TF32) != K1).nnz == 0
    assert abs(K1 - gio.lower_K(g)).max() / abs(gio.lower_K(g)).max() < TOL_TF32
    f = decks.nodal_load_vector(d)
    u, rep = s.solve(f, tol=1e-12, precision=gpu.PREC_MIXED)
    assert rep["converged"], rep
    assert gio.rel(u, g["ref_u"]) < TOL_U
    s.close()


def test_bulk_staged_spmv_gives_the_same_solve():
    """The FP32 SpMV that streams the matrix through shared memory by bulk
    copies computes the same row sums as the register-load kernel (same lanes
    per row); only the p.w partials are combined over another grid."""
    d = decks.box_hex20_lognormal(12, 12, 6, seed=5)
    f = gpu.face_load_vector(d)
    s = system(d)
    s.assemble()
    res = {}
    for bulk in (0, 1):
        s.set_option(gpu.OPT_SPMV_BULK_FP32, bulk)
        u, rep = s.solve(f, tol=1e-10, precision=gpu.PREC_MIXED)
        assert rep["converged"], rep
        res[bulk] = (u, rep)
    assert abs(res[0][1]["iterations"] - res[1][1]["iterations"]) <= 2
    assert gio.rel(res[0][0], res[1][0]) < 1e-9
    u2, _ = s.solve(f, tol=1e-10, precision=gpu.PREC_MIXED)
    assert np.array_equal(u2, res[1][0])   # deterministic
    s.close()


def test_tensor_core_path_with_tied_interfaces():
    """The four-block tied column on the tensor-core stiffness: B-spline and
    hex buckets on tcgen05, tied elements' FP64 matrices scattered into the
    FP32 blocks, FP64 residuals element by element (tied elements from their
    FP64 matrices); against the CPU elimination oracle."""
    from oracle import tie_oracle as to
    d = decks.tied_column(hex8=(4, 4, 2), hex20=(3, 3, 2), p2=(3, 3, 2), p3=(2, 2, 2), jitter=0.05, seed=3)
    f = decks.nodal_load_vector(d)
    u_o, ok, it = to.solve(d, f)
    assert ok
    s = system(d)
    s.assemble(gpu.ASM_K_TF32)
    K32 = s.lower_csr(gpu.ASM_K_TF32)
    s.assemble()
    K64 = s.lower_csr()
    assert abs(K32 - K64).max() / abs(K64).max() < TOL_TF32
    s.assemble(gpu.ASM_K_TF32)
    u, rep = s.solve(f, tol=1e-12, precision=gpu.PREC_MIXED, raise_on_nonconv=False)
    print("tied, tensor-core stiffness:", rep)
    assert rep["converged"] and rep["true_rel_residual"] < 1e-11, rep
    assert gio.rel(u, u_o) < TOL_U
    s.close()


@pytest.mark.parametrize("which", ["tied_column", "iga_p3_box", "hex20_box"])
def test_element_by_element_residual_is_the_assembled_operator(which):
    """The mixed solve on the tensor-core stiffness forms its FP64 residuals
    element by element (ties prolonged and restricted around it).  Started
    from the FP64 solve's solution, its first residual is that solution's
    residual under the assembled FP64 K, so it stops at once."""
    if which == "tied_column":
        d = decks.tied_column(hex8=(4, 4, 2), hex20=(3, 3, 2), p2=(3, 3, 2), p3=(2, 2, 2), jitter=0.05, seed=3)
        f = decks.nodal_load_vector(d)
    elif which == "iga_p3_box":
        d, _ = gio.load("iga_p3_box")
        f = decks.nodal_load_vector(d)
    else:
        d = decks.box_hex20_lognormal(6, 6, 3, seed=9)
        f = gpu.face_load_vector(d)
    s = system(d)
    s.assemble()
    u64, r64 = s.solve(f, tol=1e-13, precision=gpu.PREC_FP64, maxit=100000)
    s.assemble(gpu.ASM_K_TF32)
    u, rep = s.solve(f, tol=1e-9, precision=gpu.PREC_MIXED, u0=u64, raise_on_nonconv=False)
    print(which, "FP64 solve", r64["true_rel_residual"], "element-by-element residual at it", rep)
    assert rep["converged"] and rep["iterations"] == 0, rep
    assert rep["true_rel_residual"] < 1e-11, rep
    s.close()


@pytest.mark.parametrize("which", ["tied_column", "hex20_box", "iga_p3_box", "mixed_hex"])
def test_persistent_multi_bucket_assembly_equals_per_colour_launches(which):
    """FAST_OPT_PERSISTENT_ASSEMBLY: the regular elements of every bucket
    (hex8, hex20, B-spline p=2 / p=3) in one cooperative launch, colour k of
    every bucket as phase k.  K32 is the same bits as the per-colour launches'
    (with first-touch stores and with the zero fill), in far fewer launches,
    and the mixed solve on it converges as before."""
    if which == "tied_column":
        d = decks.tied_column(hex8=(4, 4, 2), hex20=(3, 3, 2), p2=(3, 3, 2), p3=(2, 2, 2), jitter=0.05, seed=3)
        f = decks.nodal_load_vector(d)
    elif which == "hex20_box":
        d = decks.box_hex20_lognormal(8, 8, 4, seed=4)
        f = gpu.face_load_vector(d)
    elif which == "iga_p3_box":
        d, g = gio.load("iga_p3_box")
        f = decks.nodal_load_vector(d)
    else:
        # two buckets sharing the nodes of their interface (one box, its
        # halves on the 3x3x3 and 2x2x2 rules): their phases run one after
        # the other
        import dataclasses
        d0 = decks.box_hex20_lognormal(6, 6, 4, seed=6)
        f = gpu.face_load_vector(d0)
        h = d0.num_elems // 2
        nofaces = dict(face_elem=None, face_corners=None, face_q=None, face_local=None, blocks=[])
        blk = dataclasses.replace(d0, conn=d0.conn[h:], E=d0.E[h:], nu=d0.nu[h:], ngp=(2, 2, 2), **nofaces)
        d = dataclasses.replace(d0, conn=d0.conn[:h], E=d0.E[:h], nu=d0.nu[:h], **nofaces)
        d.blocks = [blk]
    s = system(d)
    for zero_fill in (0, 1):
        s.set_option(gpu.OPT_ZERO_FILL, zero_fill)
        s.set_option(gpu.OPT_PERSISTENT_ASSEMBLY, 0)
        n0 = s.launch_count()
        s.assemble(gpu.ASM_K_TF32)
        n_col = s.launch_count() - n0
        K_col = s.lower_csr(gpu.ASM_K_TF32)
        s.set_option(gpu.OPT_PERSISTENT_ASSEMBLY, 1)
        n0 = s.launch_count()
        s.assemble(gpu.ASM_K_TF32)
        n_per = s.launch_count() - n0
        K_per = s.lower_csr(gpu.ASM_K_TF32)
        assert K_per.nnz == K_col.nnz and abs(K_per - K_col).max() == 0, (which, zero_fill)
        assert n_per < n_col or n_col <= 3, (n_per, n_col)
        print(which, "zero fill" if zero_fill else "first touch", "launches per colour %d, persistent %d"
              % (n_col, n_per))
    s.set_option(gpu.OPT_ZERO_FILL, 0)
    u, rep = s.solve(f, tol=1e-10, precision=gpu.PREC_MIXED)
    assert rep["converged"], rep
    s.close()
