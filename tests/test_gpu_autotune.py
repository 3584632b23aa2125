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
    u0, r0 = s.solve(f, tol=1e-12, precision=gpu.PREC_FP64)
    t = s.autotune()
    assert t["lanes_fp32"] in (4, 8, 16, 32) and t["lanes_fp64"] in (4, 8, 16, 32)
    assert all(v > 0 for v in t["ms_fp32_lanes_4_8_16_32"] + t["ms_fp64_lanes_4_8_16_32"])
    assert t["us_iter_persistent"] > 0 and t["us_iter_kernels"] > 0
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
