"""Device linear Newmark (fast_gpu_newmark) against the reference's own
cCtrlNewmark run (golden fixture nm_hex20_box: the unmodified `fast` binary's
printed displacements, velocities and accelerations of 20 steps)."""
import numpy as np
import pytest

from fast_b200 import gpu
from tests import golden_io as gio

pytestmark = pytest.mark.gpu


def node_field(eq, x):
    out = np.zeros(eq.shape)
    m = eq > 0
    out[m] = x[eq[m] - 1]
    return out


@pytest.mark.parametrize("precision,tol,bound", [(gpu.PREC_FP64, 1e-13, 1e-9), (gpu.PREC_MIXED, 1e-12, 1e-8)])
def test_newmark_matches_reference(precision, tol, bound):
    d, g = gio.load("nm_hex20_box")
    s = gpu.GpuSystem(0)
    s.upload(d)
    eq = g["ref_node_eq"].reshape(-1, 3)
    steps = int(g["steps"])
    (u, v, a), hist, rep = s.newmark(g["ref_f"], steps, float(g["time_step"]), float(g["gamma"]), float(g["beta"]),
                                     precision=precision, tol=tol, probes=np.arange(s.neq))
    assert rep["steps_done"] == steps and rep["failed_step"] == 0
    for k in range(steps):
        assert gio.rel(node_field(eq, hist[k]), g["ref_u_steps"][k]) < bound, k
    assert gio.rel(node_field(eq, v), g["ref_v_steps"][-1]) < 10 * bound
    assert gio.rel(node_field(eq, a), g["ref_a_steps"][-1]) < 100 * bound
    # the printout's running maxima
    assert rep["umax"] == pytest.approx(np.abs(g["ref_u_steps"]).max(), rel=1e-7)
    assert rep["vmax"] == pytest.approx(np.abs(g["ref_v_steps"]).max(), rel=1e-6)
    s.close()


def test_newmark_warm_start_saves_iterations():
    d, g = gio.load("nm_hex20_box")
    s = gpu.GpuSystem(0)
    s.upload(d)
    args = (g["ref_f"], int(g["steps"]), float(g["time_step"]))
    _, h1, r1 = s.newmark(*args, tol=1e-12, warm=True, probes=[0, 1, 2])
    _, h0, r0 = s.newmark(*args, tol=1e-12, warm=False, probes=[0, 1, 2])
    assert r1["linear_iterations"] < r0["linear_iterations"]
    np.testing.assert_allclose(h1, h0, rtol=1e-8, atol=1e-14)
    s.close()


@pytest.mark.parametrize("precision", [gpu.PREC_FP64, gpu.PREC_MIXED])
def test_newmark_graph_replay_equals_direct_launches(precision):
    """Every step after the first replays one captured CUDA graph (the PCG
    loop as a conditional WHILE node); launching kernel by kernel gives the
    same steps.  With the same kernels on both sides (the kernel-per-step PCG
    iteration, the same check interval) the steps are the same bits; the
    persistent cooperative PCG kernel, which the launched steps take for small
    systems by default, sums in another order, so that run agrees to the
    solver tolerance instead."""
    d, g = gio.load("nm_hex20_box")
    s = gpu.GpuSystem(0)
    s.upload(d)
    args = (g["ref_f"], int(g["steps"]), float(g["time_step"]))
    probes = np.arange(s.neq)
    kw = dict(precision=precision, tol=1e-12, probes=probes, check_every=16)
    (u_p, _, _), h_p, r_p = s.newmark(*args, **kw)            # graphs (the default)
    s.set_option(gpu.OPT_PERSISTENT_MAX_NODES, 0)
    (u1, _, _), h1, r1 = s.newmark(*args, **kw)
    s.set_option(gpu.OPT_GRAPH_STEPS, 0)
    (u0, _, _), h0, r0 = s.newmark(*args, **kw)
    assert r1["steps_done"] == r0["steps_done"] == r_p["steps_done"] == int(g["steps"])
    assert r1["linear_iterations"] == r0["linear_iterations"]
    assert np.array_equal(h1, h0) and np.array_equal(u1, u0)
    s.set_option(gpu.OPT_PERSISTENT_MAX_NODES, 1 << 20)
    (u2, _, _), h2, r2 = s.newmark(*args, **kw)                # launched, persistent PCG
    assert abs(r2["linear_iterations"] - r1["linear_iterations"]) <= 2 * int(g["steps"])
    assert gio.rel(h2, h1) < 1e-9 and gio.rel(u2, u1) < 1e-9
    s.close()


@pytest.mark.parametrize("precision,tol,bound", [(gpu.PREC_FP64, 1e-13, 1e-9), (gpu.PREC_MIXED, 1e-12, 1e-8)])
def test_damped_newmark_matches_reference(precision, tol, bound):
    """Rayleigh damping (%HEADER.ANALYSIS.RAYLEIGH.DAMPING): C = alpha M +
    beta K, K_eff = K + a0 M + a1 C, f_eff += C (a1 u + a4 v + a5 a), against
    the reference binary's damped run of the same box."""
    d, g = gio.load("nm_hex20_box_damped")
    s = gpu.GpuSystem(0)
    s.upload(d)
    eq = g["ref_node_eq"].reshape(-1, 3)
    steps = int(g["steps"])
    (u, v, a), hist, rep = s.newmark(g["ref_f"], steps, float(g["time_step"]), float(g["gamma"]), float(g["beta"]),
                                     precision=precision, tol=tol, probes=np.arange(s.neq),
                                     rayleigh=tuple(g["rayleigh"]))
    assert rep["steps_done"] == steps and rep["failed_step"] == 0
    for k in range(steps):
        assert gio.rel(node_field(eq, hist[k]), g["ref_u_steps"][k]) < bound, k
    assert gio.rel(node_field(eq, v), g["ref_v_steps"][-1]) < 10 * bound
    assert gio.rel(node_field(eq, a), g["ref_a_steps"][-1]) < 100 * bound
    s.close()
