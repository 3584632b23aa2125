"""Parity of the benchmarked workloads at their full size against the oracle
(fixtures made by tests/golden/make_full_size.py).

* hex20 box 64x64x32 (1,609,920 equations, lognormal E): the oracle is the
  C restatement's K (pinned to the reference's StiffMat / StiffnessMatrix at
  1e-13) solved by the reference's Jacobi PCG iteration to 1e-13.  The device
  solves with the FP64 path, the mixed path and the mixed path on the
  tensor-core stiffness, to the benchmark's 1e-8 and to 1e-10.
* TL hex8 plate 40x40x4 under pressure, 40 Newton load steps: the oracle is
  the reference's own `fast` binary (cCtrlNR) run to 1e-10; every step of the
  device Newton driver is compared.
* the four-block tied column (B-spline p=2, hex8, hex20, B-spline p=3): the
  oracle eliminates the ties on the CPU (oracle/tie_oracle.py) and solves to
  1e-13.

Each fixture holds the oracle's values at a seeded sample of entries, its
norms and seeded weighted sums over every entry; the errors below are
    e_sample = max over the sample |u - u_o| / max |u_o|
    e_check  = max_k |w_k . (u - u_o)| / (|w_k|_2 |u_o|_2)
the latter a size-independent estimate of the relative 2-norm error.
"""
import os

import numpy as np
import pytest

from fast_b200 import decks, gpu
from tests.golden import make_full_size as mfs

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# bounds on e_sample and e_check by solver tolerance: 1e-9 is the parity bar
# at 1e-10; a solve stopped at the benchmark's own 1e-8 carries the error of
# that stop, which depends on the conditioning and on where the iteration
# happened to stop: the oracle's own PCG stopped at 1e-8 is 1.0e-8 from its
# 1e-13 solution on the box (the fixture's rel_diff_1e-8), the mixed-precision
# iteration on the tied column stopped 3.5e-8 from it.  At 1e-8 the bound is
# ten times the tolerance.
BOUND = {1e-10: 1e-9, 1e-8: 1e-7}


def _fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


def errors(u, z, idx_key="idx", u_key="u_idx", checks_key="checks", norm_key="norm2", amax_key="amax"):
    u = np.asarray(u, dtype=np.float64).ravel()
    W = mfs.checksum_weights(u.size)
    e_sample = float(np.abs(u[z[idx_key]] - z[u_key]).max() / float(z[amax_key]))
    wn = np.linalg.norm(W, axis=1)
    e_check = float((np.abs(W @ u - z[checks_key]) / (wn * float(z[norm_key]))).max())
    return e_sample, e_check


@pytest.fixture(scope="module")
def box():
    z = _fixture("full_hex20_64x64x32")
    d = decks.box_hex20_lognormal(64, 64, 32, seed=0)
    f = gpu.face_load_vector(d)
    assert d.num_eq() == int(z["n"])
    assert abs(np.linalg.norm(f) - float(z["f_norm2"])) <= 1e-12 * float(z["f_norm2"])
    s = gpu.GpuSystem(0)
    s.upload(d)
    yield s, f, z
    s.close()


@pytest.mark.parametrize("tol", [1e-8, 1e-10])
@pytest.mark.parametrize("path", ["fp64", "mixed", "mixed_tf32"])
def test_full_hex20_box_against_oracle(box, path, tol):
    s, f, z = box
    if path == "mixed_tf32":
        s.assemble(gpu.ASM_K_TF32)
    else:
        s.assemble()
    prec = gpu.PREC_FP64 if path == "fp64" else gpu.PREC_MIXED
    u, rep = s.solve(f, tol=tol, precision=prec)
    assert rep["converged"] and rep["true_rel_residual"] < tol, rep
    e_sample, e_check = errors(u, z)
    print("%s tol %.0e: %d iterations, e_sample %.2e, e_check %.2e" % (path, tol, rep["iterations"], e_sample,
                                                                      e_check))
    assert e_sample < BOUND[tol] and e_check < BOUND[tol], (e_sample, e_check)


def test_full_plate_newton_against_reference_cctrlnr():
    z = _fixture("full_plate_tl_40x40x4")
    d = decks.plate_tl_hex8(40, 40, 4, L=10.0, t=1.0, pressure=40.0, steps=40, tol=1e-8)
    q = gpu.face_load_vector(d)
    s = gpu.GpuSystem(0)
    s.upload(d)
    eq = d.node_eq()
    m = eq > 0
    for prec, pred in ((gpu.PREC_FP64, gpu.PREDICT_NONE), (gpu.PREC_MIXED, gpu.PREDICT_SECANT)):
        hist, iters, rep = s.nr_solve(q, 40, 1.0 / 40, tol=1e-8, max_iter=30, predictor=pred, precision=prec,
                                      lin_tol_rel=1e-3 if prec == gpu.PREC_MIXED else 0.0, lin_tol=1e-10)
        assert rep["converged_steps"] == 40, rep
        worst = (0.0, 0.0)
        for k in range(40):
            unode = np.zeros((d.num_nodes, 3))
            unode[m] = hist[k][eq[m] - 1]
            flat = unode.ravel()
            zk = dict(idx=z["idx"], u_idx=z["u_idx"][k], checks=z["checks"][k], norm2=z["norm2"][k],
                      amax=z["amax"][k])
            es, ec = errors(flat, zk)
            worst = (max(worst[0], es), max(worst[1], ec))
        last = np.zeros((d.num_nodes, 3))
        last[m] = hist[-1][eq[m] - 1]
        e_last = float(np.abs(last - z["u_last"]).max() / np.abs(z["u_last"]).max())
        print("plate prec %d predictor %d: %d Newton iterations, worst e_sample %.2e e_check %.2e, last step "
              "(every entry) %.2e" % (prec, pred, rep["iterations"], worst[0], worst[1], e_last))
        assert worst[0] < 1e-7 and worst[1] < 1e-7 and e_last < 1e-7
    s.close()


@pytest.mark.parametrize("path", ["fp64", "mixed", "mixed_tf32"])
def test_full_tied_column_against_oracle(path):
    z = _fixture("full_tied_column")
    d = decks.tied_column()
    f = decks.nodal_load_vector(d)
    s = gpu.GpuSystem(0)
    s.upload(d)
    s.assemble(gpu.ASM_K_TF32 if path == "mixed_tf32" else gpu.ASM_K)
    prec = gpu.PREC_FP64 if path == "fp64" else gpu.PREC_MIXED
    for tol in (1e-8, 1e-10):
        u, rep = s.solve(f, tol=tol, precision=prec)
        assert rep["converged"], rep
        e_sample, e_check = errors(u, z)
        print("tied %s tol %.0e: %d iterations, e_sample %.2e, e_check %.2e" % (path, tol, rep["iterations"],
                                                                               e_sample, e_check))
        assert e_sample < BOUND[tol] and e_check < BOUND[tol], (e_sample, e_check)
    s.close()
