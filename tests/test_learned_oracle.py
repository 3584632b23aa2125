"""CPU checks of the learned predictor's oracle (oracle/mlp_oracle.py): its
gradients against central finite differences, its BF16 rounding, its POD
basis and its sample construction.  No device is used."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 3.0e-3, 0.0], np.float32)
    r = mo.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa -> 1
    # 1 + 3*2^-8 is a tie between 1 + 2^-7 and 1 + 2^-6: even -> 1 + 2^-6
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0 ** -6 and r[3] == 1.0
    assert r[4] == -2.5 and r[6] == 0.0
    assert abs(r[5] - 3.0e-3) <= 3.0e-3 * 2.0 ** -8


def test_bf16_relative_error_bound():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-5, 5, 10000)
    r = mo.bf16(x)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8 * (1 + 1e-7))


@pytest.mark.parametrize("dims", [[7, 5, 3], [9, 6, 6, 4], [129, 16, 16, 32]])
def test_oracle_gradient_matches_finite_differences(dims):
    rng = np.random.default_rng(len(dims))
    net = mo.Mlp(dims)
    n = sum(o * i + o for i, o in zip(dims[:-1], dims[1:]))
    p = rng.standard_normal(n) * 0.3
    x = rng.standard_normal((11, dims[0]))
    t = rng.standard_normal((11, dims[-1]))
    _, g = net.loss_grad(p, x, t)
    idx = rng.choice(n, size=min(n, 60), replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(n)
        e[i] = h
        fd = (net.loss_grad(p + e, x, t)[0] - net.loss_grad(p - e, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(g[i]), (i, fd, g[i])


def test_emulated_gradient_close_to_exact():
    rng = np.random.default_rng(5)
    dims = [129, 64, 64, 32]
    net = mo.Mlp(dims)
    n = sum(o * i + o for i, o in zip(dims[:-1], dims[1:]))
    p = rng.standard_normal(n) * 0.1
    x = rng.standard_normal((40, 129))
    t = rng.standard_normal((40, 32))
    _, g = net.loss_grad(p, x, t)
    _, ge = net.loss_grad(p, x, t, emulate=True)
    assert np.linalg.norm(ge - g) / np.linalg.norm(g) < 2e-2


def test_pod_basis_recovers_low_rank():
    rng = np.random.default_rng(2)
    U = np.linalg.qr(rng.standard_normal((500, 6)))[0]
    C = rng.standard_normal((40, 6)) * np.array([100, 30, 10, 3, 1, 0.3])
    S = C @ U.T
    phi, energy = mo.pod_basis(S, 6)
    assert energy == pytest.approx(1.0, abs=1e-12)
    s = np.linalg.svd(phi.T @ U, compute_uv=False)
    assert np.all(s > 1 - 1e-10)


def test_samples_targets_are_secant_misses():
    # a trajectory with coefficients quadratic in the load factor: the secant
    # miss is the constant second difference
    lam = np.arange(1, 11) / 10.0
    A = np.stack([3 * lam ** 2, -lam ** 2 + lam], axis=1)
    X, T = mo.samples([A], [lam], history=3, modes=2)
    assert X.shape == (9, 7) and T.shape == (9, 2)
    np.testing.assert_allclose(T[1:], np.tile([3 * 0.02, -0.02], (8, 1)), atol=1e-14)
    # step 2: latest set a_1, increments a_1 - a_0 = a_1 and a_0 - a_{-1} = 0
    np.testing.assert_allclose(X[0, 1:3], A[0])
    np.testing.assert_allclose(X[0, 3:5], A[0])
    np.testing.assert_allclose(X[0, 5:], 0.0)
    # later steps: the state and its backward differences
    np.testing.assert_allclose(X[5, 1:3], A[5])
    np.testing.assert_allclose(X[5, 3:5], A[5] - A[4])
    np.testing.assert_allclose(X[5, 5:7], A[4] - A[3])
