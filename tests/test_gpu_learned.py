"""GPU checks of the learned load-step predictor against its CPU oracle
(oracle/mlp_oracle.py): the tcgen05 BF16 GEMM, the MLP forward pass and
gradients, the POD basis, the training samples, and what the trained
predictor gains in a Newton solve over the secant start it competes with."""
import numpy as np
import pytest

from fast_b200 import decks, gpu, learned
from oracle import mlp_oracle as mo
from tests import golden_io as gio

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    s = gpu.GpuSystem(0)
    yield s
    s.close()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("M,N,K", [(1, 32, 129), (128, 64, 64), (130, 200, 70), (300, 129, 2496), (257, 256, 256),
                                   (5, 8, 3)])
@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
def test_tensor_core_gemm_matches_bf16_oracle(system, M, N, K, ta, tb):
    rng = np.random.default_rng(M * 7 + N * 3 + K + 2 * ta + tb)
    A = rng.standard_normal((K, M) if ta else (M, K)).astype(np.float32)
    B = rng.standard_normal((K, N) if tb else (N, K)).astype(np.float32)
    C = system.mlp_gemm(A, B, ta, tb)
    Ar = mo.bf16(A.T if ta else A)
    Br = mo.bf16(B.T if tb else B)
    ref = Ar @ Br.T
    # FP32 accumulation of exact BF16 products: error ~ sqrt(K) * 2^-24 * |a||b|
    bound = 2e-5 * np.sqrt(K) * (np.abs(Ar) @ np.abs(Br).T) + 1e-30
    assert np.all(np.abs(C - ref) <= bound), float(np.max(np.abs(C - ref) / bound))
    # and the BF16 operands cost about 2^-8 relative against exact FP32 operands
    exact = (A.T if ta else A).astype(np.float64) @ (B.T if tb else B).astype(np.float64).T
    assert rel(C, exact) < 1e-2


@pytest.fixture(scope="module")
def small_plate(system):
    d = decks.plate_tl_hex8(10, 10, 2, L=10.0, t=1.0, pressure=60.0, steps=16, tol=1e-8)
    system.upload(d)
    q = gpu.face_load_vector(d)
    return d, q


@pytest.fixture(scope="module")
def predictor(system, small_plate):
    d, q = small_plate
    p, info = learned.train_predictor(system, d, q, variants=12, seed=3, steps=16, modes=16, history=4, width=64,
                                      hidden=2, epochs=1500, lr=3e-3)
    yield p, info
    p.close()


@pytest.mark.parametrize("batch", [300, 2496])
def test_mlp_forward_and_gradients_match_oracle(system, small_plate, batch):
    # batch 2496 (the training batch) takes the split-K weight-gradient GEMMs
    dims = [129, 256, 256, 32]
    p = gpu.LearnedPredictor(system, modes=32, history=4, width=256, hidden=2, seed=11)
    try:
        assert p.dims() == dims
        net = mo.Mlp(dims)
        rng = np.random.default_rng(4)
        params = (rng.standard_normal(p.params().size) * 0.08).astype(np.float32)
        p.params(set_to=params)
        x = rng.standard_normal((batch, 129)).astype(np.float32)
        t = rng.standard_normal((batch, 32)).astype(np.float32)
        y = p.forward(x)
        ye = net.forward(params, x, emulate=True)[-1]
        assert rel(y, ye) < 1e-4
        loss, g = p.loss_grad(x, t)
        le, ge = net.loss_grad(params, x, t, emulate=True)
        lx, gx = net.loss_grad(params, x, t)
        assert abs(loss - le) <= 1e-4 * le
        # per parameter block against the BF16-emulating oracle, then the exact FP64 oracle
        off = 0
        for i, o in zip(dims[:-1], dims[1:]):
            for size in (o * i, o):
                blk = slice(off, off + size)
                # BF16 rounding of slightly different FP32 values flips a few operands
                assert rel(g[blk], ge[blk]) < 1e-3, (i, o, size)
                assert rel(g[blk], gx[blk]) < 3e-2, (i, o, size)
                off += size
    finally:
        p.close()


@pytest.mark.parametrize("dims_key", ["129-256-256-32", "65-64-64-16"])
def test_single_row_forward_matches_batched_forward(system, small_plate, dims_key):
    """The single-row CUDA-core forward the predictor runs (batch 1) against
    the tcgen05 batched forward of the same rows and the BF16-emulating
    oracle; the same bits on every call."""
    dims = [int(v) for v in dims_key.split("-")]
    p = gpu.LearnedPredictor(system, modes=dims[-1], history=(dims[0] - 1) // dims[-1], width=dims[1],
                             hidden=len(dims) - 2, seed=5)
    try:
        assert p.dims() == dims
        net = mo.Mlp(dims)
        rng = np.random.default_rng(9)
        params = (rng.standard_normal(p.params().size) * 0.08).astype(np.float32)
        p.params(set_to=params)
        x = rng.standard_normal((6, dims[0])).astype(np.float32)
        yb = p.forward(x)
        ye = net.forward(params, x, emulate=True)[-1]
        for i in range(x.shape[0]):
            y1 = p.forward(x[i:i + 1])
            # a BF16 rounding of a hidden activation may flip between the two
            # summation orders, as it does against the oracle
            assert rel(y1[0], yb[i]) < 1e-4, i
            assert rel(y1[0], ye[i]) < 1e-4, i
            assert np.array_equal(y1, p.forward(x[i:i + 1]))
    finally:
        p.close()


def test_pod_basis_matches_dense_svd(system, small_plate, predictor):
    d, q = small_plate
    p, info = predictor
    phi = p.basis()
    k = phi.shape[1]
    # the same snapshots, regenerated
    snaps = np.concatenate([h for _, h, _ in learned.trajectories(system, d, q, 12, seed=3, steps=16)])
    ref, energy = mo.pod_basis(snaps, k)
    assert info["captured_energy"] == pytest.approx(energy, rel=1e-6)
    np.testing.assert_allclose(phi.T @ phi, np.eye(k), atol=1e-10)
    # what the basis leaves out of the snapshots is what the dense SVD's leaves out
    res = np.linalg.norm(snaps - (snaps @ phi) @ phi.T) ** 2 / np.linalg.norm(snaps) ** 2
    assert res == pytest.approx(1 - energy, rel=1e-3, abs=1e-13)
    # and the leading modes span the same space
    s = np.linalg.svd(phi[:, :4].T @ ref[:, :4], compute_uv=False)
    assert np.all(s > 1 - 1e-6), s


def test_training_samples_match_oracle(system, small_plate, predictor):
    d, q = small_plate
    p, _ = predictor
    phi = p.basis()
    k = phi.shape[1]
    coef, lams = [], []
    for lam, h, _ in learned.trajectories(system, d, q, 12, seed=3, steps=16):
        coef.append(h @ phi)
        lams.append(lam)
    X, T = mo.samples(coef, lams, history=4, modes=16)
    A = np.concatenate(coef)
    sigma = np.sqrt(np.mean(A ** 2, axis=0))
    delta = np.sqrt(np.mean(X[:, 17:33] ** 2, axis=0))
    tau = np.sqrt(np.mean(T ** 2, axis=0))
    xs, ts = p.samples()
    assert xs.shape == X.shape and ts.shape == T.shape
    np.testing.assert_allclose(xs[:, 0], X[:, 0], rtol=1e-6)
    np.testing.assert_allclose(xs[:, 1:17], X[:, 1:17] / sigma, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(xs[:, 17:], X[:, 17:] / np.tile(delta, 3), rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(ts, T / tau, rtol=1e-4, atol=1e-4)


def test_training_reduces_loss(predictor):
    _, info = predictor
    r = info["report"]
    assert info["converged_variants"] == 12
    assert r["samples"] == 12 * 15 and r["params"] > 0
    assert info["last_loss"] < 0.05 * info["first_loss"], info


def _solve_variant(system, d, q, seed, **kw):
    ps, E = decks.plate_variant_params(seed, d.num_elems)
    system.update_material(E=E)
    try:
        return system.nr_solve(ps * q, 16, 1 / 16, tol=1e-8, max_iter=30, precision=gpu.PREC_FP64, lin_tol=1e-12,
                               **kw)
    finally:
        system.update_material(E=d.E)


def test_device_features_match_training_samples(system, small_plate, predictor):
    """The features the predictor builds on the device from its coefficient
    ring equal the training sample of the same trajectory and step."""
    d, q = small_plate
    p, _ = predictor
    p.configure(use_network=True, galerkin_iters=0)
    _, _, r = _solve_variant(system, d, q, 3 * 100003 + 0, learned=p)
    assert r["converged_steps"] == 16
    xs, _ = p.samples()
    np.testing.assert_allclose(p.last_input(), xs[14], rtol=1e-3, atol=1e-4)


def test_learned_start_beats_secant_on_unseen_variant(system, small_plate, predictor):
    """What the network gains: on a held-out variant the network's start is
    accepted over the secant start at most steps, and Newton needs fewer
    iterations than with the secant start alone; both reach the same
    tolerance and the same displacements."""
    d, q = small_plate
    p, _ = predictor
    p.configure(use_network=True, galerkin_iters=0)
    h0, _, r0 = _solve_variant(system, d, q, 999, predictor=gpu.PREDICT_SECANT)
    h1, _, r1 = _solve_variant(system, d, q, 999, learned=p)
    h2, _, r2 = _solve_variant(system, d, q, 999, predictor=gpu.PREDICT_NONE)
    assert r0["converged_steps"] == r1["converged_steps"] == r2["converged_steps"] == 16
    assert r1["predictions"] == 15
    assert r1["predictions_accepted"] >= 12, r1
    assert r1["iterations"] < r0["iterations"] <= r2["iterations"], (r1, r0, r2)
    assert rel(h1[-1], h2[-1]) < 1e-6 and rel(h0[-1], h2[-1]) < 1e-6


def test_galerkin_refined_start(system, small_plate, predictor):
    """One reduced (POD-Galerkin) Newton correction of the network's start:
    accepted at every step, fewer Newton iterations than the unrefined
    network start and than the refined secant start (the network's gain)."""
    d, q = small_plate
    p, _ = predictor
    try:
        p.configure(use_network=True, galerkin_iters=0)
        _, _, r_net = _solve_variant(system, d, q, 999, learned=p)
        p.configure(use_network=False, galerkin_iters=1)
        _, _, r_sec = _solve_variant(system, d, q, 999, learned=p)
        p.configure(use_network=True, galerkin_iters=1)
        h, _, r_both = _solve_variant(system, d, q, 999, learned=p)
        h_ref, _, r_none = _solve_variant(system, d, q, 999, predictor=gpu.PREDICT_NONE)
    finally:
        p.configure(use_network=True, galerkin_iters=0)
    assert r_both["converged_steps"] == 16 and r_both["predictions_accepted"] == 15, r_both
    assert r_both["iterations"] < r_net["iterations"], (r_both, r_net)
    assert r_both["iterations"] <= r_sec["iterations"], (r_both, r_sec)
    assert r_both["iterations"] < r_none["iterations"]
    assert rel(h[-1], h_ref[-1]) < 1e-6


def test_predictor_spans_are_timed(system, small_plate, predictor):
    """Live timing covers the predictor's two phases, the internal forces and
    the linear solves of a Newton run."""
    d, q = small_plate
    p, _ = predictor
    try:
        p.configure(use_network=True, galerkin_iters=1)
        system.kernel_timing(True)
        _, _, r = _solve_variant(system, d, q, 999, learned=p)
        st = {k: system.kernel_stats(k) for k in (gpu.KERNEL_PREDICT_NET, gpu.KERNEL_PREDICT_GALERKIN,
                                                  gpu.KERNEL_INTERNAL_FORCE, gpu.KERNEL_LINEAR_SOLVE)}
    finally:
        system.kernel_timing(False)
        p.configure(use_network=True, galerkin_iters=0)
    assert st[gpu.KERNEL_PREDICT_NET][0] == 15 and st[gpu.KERNEL_PREDICT_GALERKIN][0] == 15
    assert st[gpu.KERNEL_LINEAR_SOLVE][0] == r["iterations"]
    assert st[gpu.KERNEL_INTERNAL_FORCE][0] >= r["iterations"] + 15
    assert all(v[1] > 0 for v in st.values())


def test_training_trajectories_are_the_reference_cctrlnr_paths():
    """The predictor trains on load-step trajectories of seeded pressure /
    stiffness variants (fast_b200.learned.trajectories, the device Newton
    driver).  On two such variants of a small plate those trajectories are the
    ones the reference's own cCtrlNR computes (the `fast` binary run on the
    same variant decks, every step)."""
    from fast_b200 import learned
    d, g = gio.load("nr_plate_variants")
    q = gpu.face_load_vector(d)
    s = gpu.GpuSystem(0)
    s.upload(d)
    eq = d.node_eq()
    m = eq > 0
    got = list(learned.trajectories(s, d, q, int(g["variants"]), seed=0, steps=int(g["steps"]), tol=float(g["tol"]),
                                    max_iter=int(g["maxit"]), precision=gpu.PREC_FP64))
    assert len(got) == int(g["variants"])
    for v, (lam, h, rep) in enumerate(got):
        for k in range(h.shape[0]):
            un = np.zeros((d.num_nodes, 3))
            un[m] = h[k][eq[m] - 1]
            assert gio.rel(un, g["ref_u_steps"][v][k]) < 1e-8, (v, k)
    s.close()
