"""GMRES(m) of the matrix-free implicit stepper (ablate_b200.implicit.gmres) on CPU tensors."""
import numpy as np
import pytest


@pytest.mark.parametrize("restart", [5, 30])
def test_gmres_solves_a_nonsymmetric_system(restart):
    torch = pytest.importorskip("torch")
    from ablate_b200.implicit import gmres
    rng = np.random.default_rng(0)
    n = 120
    A = np.eye(n) + 0.4 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal((n // 4, 4))  # vectors keep the (rows, components) shape of a state
    At = torch.from_numpy(A)

    def apply(v):
        return (At @ v.reshape(-1)).reshape(v.shape)

    x, its, res = gmres(apply, torch.from_numpy(b), restart=restart, rtol=1e-10)
    ref = np.linalg.solve(A, b.reshape(-1)).reshape(b.shape)
    assert res <= 1e-10 * np.linalg.norm(b)
    np.testing.assert_allclose(x.numpy(), ref, rtol=0, atol=1e-8 * np.abs(ref).max())
    assert its <= (n if restart == 30 else 10 * n)


def test_gmres_exact_after_n_iterations_without_restart():
    torch = pytest.importorskip("torch")
    from ablate_b200.implicit import gmres
    rng = np.random.default_rng(1)
    n = 20
    A = rng.standard_normal((n, n)) + 5 * np.eye(n)
    b = rng.standard_normal(n)
    At = torch.from_numpy(A)
    x, its, res = gmres(lambda v: At @ v, torch.from_numpy(b), restart=n, rtol=1e-13)
    assert its <= n
    np.testing.assert_allclose(A @ x.numpy(), b, atol=1e-11)


def test_gmres_zero_right_hand_side():
    torch = pytest.importorskip("torch")
    from ablate_b200.implicit import gmres
    x, its, res = gmres(lambda v: 2 * v, torch.zeros(7, 3, dtype=torch.float64))
    assert its == 0 and res == 0.0 and float(x.abs().max()) == 0.0
