"""Gauss-point strains and stresses on the device (fast_gpu_gauss_stress)
against the reference's cElement::IntPntStress at its own solution.  Needs a
B200."""
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
