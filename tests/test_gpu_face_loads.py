"""Face tractions integrated on the device (fast_gpu_set_face_loads,
fast_gpu_face_load_device) against the reference's load vectors and the host
integrator, also after the coordinates move.  Needs a B200."""
import dataclasses

import numpy as np
import pytest
import torch

from fast_b200 import gpu
from tests import golden_io as gio

pytestmark = pytest.mark.gpu

CASES = [n for n in gio.names() if not n.startswith(("nr_", "iga_", "arc_", "modal_"))]


def device_f(s, scale=1.0):
    d_f = torch.full((s.neq,), 7.0, dtype=torch.float64, device="cuda")  # overwritten entirely
    s.face_load_device(d_f.data_ptr(), scale)
    s.synchronize()
    return d_f.cpu().numpy()


@pytest.mark.parametrize("name", CASES)
def test_device_face_loads_match_reference(name):
    d, g = gio.load(name)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.set_face_loads(d)
    f1 = device_f(s)
    assert gio.rel(f1, g["ref_f"]) < 1e-13
    assert gio.rel(f1, gpu.face_load_vector(d)) < 1e-14
    f2 = device_f(s, 0.5)
    assert np.array_equal(f2, 0.5 * f1) and np.array_equal(device_f(s), f1)
    s.close()


def test_device_face_loads_follow_new_coordinates():
    d, g = gio.load("cfg_hex20_lognormal_4x4x2")
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.set_face_loads(d)
    rng = np.random.default_rng(5)
    moved = dataclasses.replace(d, coords=d.coords + 0.02 * rng.standard_normal(d.coords.shape))
    s.update_coords(moved.coords)
    assert gio.rel(device_f(s), gpu.face_load_vector(moved)) < 1e-14
    s.close()
