"""The autotuner (fast_gpu_autotune) and the SpMV lane options: every launch
shape gives the same solution.  Needs a B200."""
import numpy as np
import pytest

from fast_b200 import decks, gpu
from oracle import fem_oracle as fo
from tests import golden_io as gio

pytestmark = pytest.mark.gpu


def test_autotune_choices_and_solution():
    d = decks.box_hex20_lognormal(8, 8, 4, seed=11)
    f = gpu.face_load_vector(d)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    K0 = s.lower_csr()
    u0, r0 = s.solve(f, tol=1e-12, precision=gpu.PREC_FP64)
    t = s.autotune()
    assert t["lanes_fp32"] in (4, 8, 16, 32) and t["lanes_fp64"] in (4, 8, 16, 32)
    assert all(v > 0 for v in t["ms_fp32_lanes_4_8_16_32"] + t["ms_fp64_lanes_4_8_16_32"])
    assert t["us_iter_persistent"] > 0 and t["us_iter_kernels"] > 0
    # element launch shapes: one bucket (hex20), timed on both paths
    assert len(t["elements"]) == 1 and t["elements_tensor_core_timed"]
    el = t["elements"][0]
    assert el["ms_default"] > 0 and 0 < el["ms_tuned"] <= el["ms_default"]
    assert el["tc_ms_default"] > 0 and 0 < el["tc_ms_tuned"] <= el["tc_ms_default"]
    # K is rebuilt after the timed assemblies: the same matrix, bit for bit
    assert (s.lower_csr() != K0).nnz == 0
    for prec in (gpu.PREC_FP64, gpu.PREC_MIXED):
        u, r = s.solve(f, tol=1e-12, precision=prec)
        assert r["converged"] and gio.rel(u, u0) < 1e-9
    s.close()


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_every_lane_count_solves(lanes):
    d = decks.box_hex20_lognormal(4, 4, 2, seed=7)
    f = gpu.face_load_vector(d)
    u_o, ok, it, err = fo.pcg(fo.assemble(d), f, 1e-13, 100000)
    s = gpu.GpuSystem(0)
    s.set_option(gpu.OPT_SPMV_LANES_FP32, lanes)
    s.set_option(gpu.OPT_SPMV_LANES_FP64, lanes)
    s.set_option(gpu.OPT_PERSISTENT_MAX_NODES, 0)  # the kernels the lanes apply to
    s.upload(d)
    s.assemble()
    for prec in (gpu.PREC_FP64, gpu.PREC_MIXED):
        u, r = s.solve(f, tol=1e-12, precision=prec)
        assert r["converged"] and gio.rel(u, u_o) < 1e-9
    s.close()


def test_lane_option_rejects_bad_values():
    s = gpu.GpuSystem(0)
    with pytest.raises(gpu.FastGpuError):
        s.set_option(gpu.OPT_SPMV_LANES_FP32, 12)
    s.close()


def test_every_element_launch_shape_gives_the_same_stiffness():
    """The tied column has hex8, hex20 and B-spline p=2 / p=3 buckets; every
    resident-CTA cap, every B-spline split and every tensor-core cap leaves K
    (FP64 and FP32) bit-identical, and the autotuner's choices keep it too."""
    d = decks.tied_column()
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    K0 = s.lower_csr()
    s.assemble(gpu.ASM_K_TF32)
    K0_32 = s.lower_csr(gpu.ASM_K_TF32)
    nb = s.nbuckets
    assert nb == 4
    kinds = [bk.kind for bk in d.buckets()]
    for b in range(nb):
        shapes = [(1, 0, 1, 0), (2, 1, 2, 0), (1, 2, 1, 0), (3, 4, 0, 0)]
        if kinds[b] in ("hex8", "hex20"):
            shapes += [(0, 0, 0, 1), (1, 0, 0, 1), (2, 0, 0, 1)]   # one warp per element
        for ctas, split, tc, kern in shapes:
            s.set_option(gpu.OPT_ELEM_SHAPE, gpu.elem_shape(b, ctas, split, tc, kern))
            s.assemble()
            assert (s.lower_csr() != K0).nnz == 0, (b, ctas, split, kern)
            s.assemble(gpu.ASM_K_TF32)
            assert (s.lower_csr(gpu.ASM_K_TF32) != K0_32).nnz == 0, (b, tc)
        s.set_option(gpu.OPT_ELEM_SHAPE, gpu.elem_shape(b))
    s.assemble()
    t = s.autotune()
    assert len(t["elements"]) == nb
    assert (s.lower_csr() != K0).nnz == 0
    s.assemble(gpu.ASM_K_TF32)
    assert (s.lower_csr(gpu.ASM_K_TF32) != K0_32).nnz == 0
    print(t["elements"])
    s.close()


def test_element_shape_option_rejects_a_missing_bucket():
    d = decks.box_hex20_lognormal(2, 2, 1, seed=1)
    s = gpu.GpuSystem(0)
    s.upload(d)
    with pytest.raises(gpu.FastGpuError):
        s.set_option(gpu.OPT_ELEM_SHAPE, gpu.elem_shape(5, 1))
    s.close()


@pytest.mark.parametrize("lanes", [8, 16])
def test_streaming_spmv_gives_the_same_bits(lanes):
    """FAST_OPT_SPMV_STREAM_FP32: the FP32 SpMV with cache-streaming matrix
    loads does the same arithmetic in the same order as the plain one, so the
    mixed solve returns the same bits."""
    d = decks.box_hex20_lognormal(10, 10, 5, seed=8)
    f = gpu.face_load_vector(d)
    s = gpu.GpuSystem(0)
    s.set_option(gpu.OPT_PERSISTENT_MAX_NODES, 0)   # the kernels the option applies to
    s.set_option(gpu.OPT_SPMV_LANES_FP32, lanes)
    s.upload(d)
    s.assemble()
    u0, r0 = s.solve(f, tol=1e-10, precision=gpu.PREC_MIXED)
    s.set_option(gpu.OPT_SPMV_STREAM_FP32, 1)
    u1, r1 = s.solve(f, tol=1e-10, precision=gpu.PREC_MIXED)
    assert r0["converged"] and r1["iterations"] == r0["iterations"]
    assert np.array_equal(u0, u1)
    s.close()


@pytest.mark.parametrize("ng", [(2, 2, 2), (3, 3, 3)])
def test_warp_per_element_stiffness_matches_reference(ng):
    """The FP64 hex stiffness with one warp per element gives the same K, bit
    for bit, as the CTA-per-element kernel (same arithmetic in the same
    order), and so the reference's K (hex20 lognormal box, first-touch
    stores)."""
    d = decks.box_hex20_lognormal(6, 6, 3, seed=12)
    d.ngp = ng
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble()
    K0 = s.lower_csr()
    s.set_option(gpu.OPT_ELEM_SHAPE, gpu.elem_shape(0, kernel=1))
    n0 = s.launch_count()
    s.assemble()
    K1 = s.lower_csr()
    assert K1.nnz == K0.nnz and abs(K1 - K0).max() == 0
    K = fo.assemble(d)
    R = fo_lower(K)
    assert abs(K1 - R).max() / abs(R).max() < 1e-12
    s.close()


def fo_lower(K):
    import scipy.sparse as sp
    return sp.tril(K).tocsr()


@pytest.mark.parametrize("lanes", [8, 16])
def test_col16_spmv_gives_the_same_bits(lanes):
    """FAST_OPT_SPMV_COL16_FP32: 16-bit column offsets from each row's smallest
    column (rows of this box span far fewer than 65,536 nodes) give the same
    gathers, so the mixed solve returns the same bits."""
    d = decks.box_hex20_lognormal(10, 10, 5, seed=8)
    f = gpu.face_load_vector(d)
    s = gpu.GpuSystem(0)
    s.set_option(gpu.OPT_PERSISTENT_MAX_NODES, 0)   # the kernels the option applies to
    s.set_option(gpu.OPT_SPMV_LANES_FP32, lanes)
    s.upload(d)
    s.assemble()
    u0, r0 = s.solve(f, tol=1e-10, precision=gpu.PREC_MIXED)
    s.set_option(gpu.OPT_SPMV_COL16_FP32, 1)
    u1, r1 = s.solve(f, tol=1e-10, precision=gpu.PREC_MIXED)
    assert r0["converged"] and r1["iterations"] == r0["iterations"]
    assert np.array_equal(u0, u1)
    s.close()
