"""Full-size oracle pins for the three benchmarked single-problem workloads
(TEST INFRASTRUCTURE ONLY).

    FAST_REF=<reference tree> python tests/golden/make_full_size.py plate
        TL (St. Venant-Kirchhoff) hex8 plate 40x40x4, pressure 40 over 40 load
        steps: the reference's own unmodified `fast` binary (cCtrlNR,
        ctrl/ctrlnr.cpp:47-270; skyline Crout, banded node numbering) run to
        |r|/max(1,|f|) < 1e-10, every printed step read back from its .pos file.
    python tests/golden/make_full_size.py box
        hex20 box 64x64x32 (131,072 elements, 1,609,920 equations), lognormal E
        (median 1000, sigma 0.5, seed 0): K from the C restatement of the
        reference's element stiffness (oracle/fem_oracle.c, itself pinned to the
        reference's StiffMat / StiffnessMatrix dumps at 1e-13), load from the
        restated face-load integration, then Jacobi PCG (the reference's
        PCGSolver iteration, mlib/sysmat.cpp:1061-1125) run on all host threads
        to |r|/|f| < 1e-13.
    python tests/golden/make_full_size.py tied
        the four-block tied column (B-spline p=2, hex8, hex20, B-spline p=3):
        element matrices from the restatements, ties eliminated as
        oracle/tie_oracle.py does, the reduced system solved by Jacobi PCG to
        |r|/|f| < 1e-13.

A full displacement vector is too large to commit, so each fixture stores
what a size-independent comparison needs: the oracle's displacements at a
seeded sample of entries (and every entry for the plate's last step), their
2-norm and largest magnitude, and seeded weighted sums sum_i w_i u_i over
every entry (w_i uniform in [-1, 1] from a recorded seed), which an error
anywhere in the vector moves.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from fast_b200 import decks  # noqa: E402
from oracle import refdump  # noqa: E402

SAMPLE = 32768      # sampled entries per vector
SAMPLE_STEPS = 2048 # sampled entries per load step of the Newton plate
CHECK_SEED = 12345  # seed of the checksum weights
NCHECK = 4          # independent weighted sums


def sample_index(n: int, seed: int = 7, size: int = SAMPLE) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(size, n), replace=False)).astype(np.int64)


def checksum_weights(n: int) -> np.ndarray:
    """[NCHECK][n] weights uniform in [-1, 1]; the tests regenerate them."""
    return np.random.default_rng(CHECK_SEED).uniform(-1.0, 1.0, size=(NCHECK, n))


def summary(u: np.ndarray) -> dict:
    u = np.asarray(u, dtype=np.float64).ravel()
    idx = sample_index(u.size)
    return dict(n=np.array(u.size), idx=idx, u_idx=u[idx], norm2=np.array(np.linalg.norm(u)),
                amax=np.array(np.abs(u).max()), checks=checksum_weights(u.size) @ u)


def plate():
    fast_ref = os.environ.get("FAST_REF", "")
    if not os.path.isdir(fast_ref):
        sys.exit("set FAST_REF to the reference FAST source tree")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"FAST_REF={fast_ref}", "ref"], check=True)
    d = decks.plate_tl_hex8(40, 40, 4, L=10.0, t=1.0, pressure=40.0, steps=40, tol=1e-10, maxit=30)
    tmp = tempfile.mkdtemp(prefix="full_plate_")
    base = os.path.join(tmp, "plate_40x40x4")
    decks.write_dat(d, base)
    t0 = time.time()
    subprocess.run([refdump.FAST, base, "-silent"], check=True, stdout=subprocess.DEVNULL)
    secs = time.time() - t0
    save_plate(d, base + ".pos", secs)


def save_plate(d, pos_path, secs):
    us = decks.read_pos_displacements(pos_path)               # [steps][nnode][3]
    assert us.shape[0] == 40, us.shape
    flat = us.reshape(us.shape[0], -1)
    out = dict(steps=np.array(40), pressure=np.array(40.0), ref_tol=np.array(1e-10), ref_seconds=np.array(secs),
               u_last=us[-1], centre_w=us[:, _centre_node(d), 2])
    idx = sample_index(flat.shape[1], size=SAMPLE_STEPS)
    out.update(idx=idx, u_idx=flat[:, idx], norm2=np.linalg.norm(flat, axis=1), amax=np.abs(flat).max(axis=1),
               checks=flat @ checksum_weights(flat.shape[1]).T)
    np.savez_compressed(os.path.join(HERE, "full_plate_tl_40x40x4.npz"), **out)
    print("plate: reference cCtrlNR %.1f s, centre w at the last step %.6f" % (secs, out["centre_w"][-1]))


def _centre_node(d) -> int:
    c = np.array([5.0, 5.0, 1.0])
    return int(np.argmin(np.linalg.norm(d.coords - c[None, :], axis=1)))


def _pcg_all_threads(K, f, tol, maxit=200000):
    """The reference's Jacobi PCG iteration with its SpMV and vector
    operations on all host threads (the oracle's C checker); returns u,
    iterations, recurrence error."""
    from oracle import fem_oracle as fo
    return fo.pcg_threaded(K, f, tol, maxit)


def box():
    from oracle import fem_oracle as fo
    t0 = time.time()
    d = decks.box_hex20_lognormal(64, 64, 32, seed=0)
    f = fo.face_loads(d)
    K = fo.assemble_chunked(d)
    t1 = time.time()
    u, it, err = _pcg_all_threads(K, f, 1e-13)
    t2 = time.time()
    true_res = np.linalg.norm(f - K @ u) / np.linalg.norm(f)
    out = summary(u)
    out.update(f_norm2=np.array(np.linalg.norm(f)), iterations=np.array(it), rec_err=np.array(err),
               true_rel_residual=np.array(true_res), nnz=np.array(K.nnz))
    # iteration counts of the reference's PCGSolver algorithm at the
    # benchmark's tolerance and at 1e-10, and the distance of those solutions
    # from the 1e-13 one (how far a solve stopped there is from the oracle)
    for tol, key in ((1e-8, "1e-8"), (1e-10, "1e-10")):
        ut, itt, _ = _pcg_all_threads(K, f, tol)
        out["iterations_" + key] = np.array(itt)
        out["rel_diff_" + key] = np.array(np.abs(ut - u).max() / np.abs(u).max())
    np.savez_compressed(os.path.join(HERE, "full_hex20_64x64x32.npz"), **out)
    print("box: assembled in %.0f s (nnz %d), PCG %d iterations in %.0f s, true |f-Ku|/|f| %.2e"
          % (t1 - t0, K.nnz, it, t2 - t1, true_res))


def tied():
    from oracle import tie_oracle
    t0 = time.time()
    d = decks.tied_column()
    u, info = tie_oracle.solve_full(d, tol=1e-13)
    out = summary(u)
    out.update({k: np.array(v) for k, v in info.items()})
    np.savez_compressed(os.path.join(HERE, "full_tied_column.npz"), **out)
    print("tied: %.0f s" % (time.time() - t0), info)


if __name__ == "__main__":
    what = sys.argv[1:] or ["plate", "box", "tied"]
    for w in what:
        {"plate": plate, "box": box, "tied": tied}[w]()
