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


class _LinearProblem:
    """F(U) = A U on the owned rows of a CPU tensor (3 rows of 'ghosts' copied from the first rows)."""

    def __init__(self, n=40, nc=3, seed=2):
        rng = np.random.default_rng(seed)
        self.n, self.nc = n, nc
        self.A = -np.eye(n * nc) + 0.3 * rng.standard_normal((n * nc, n * nc)) / np.sqrt(n * nc)


def _stepper(problem, dt, torch):
    from ablate_b200.implicit import BDFStepper
    A = torch.from_numpy(problem.A)
    n, nc = problem.n, problem.nc

    class Fake(BDFStepper):
        def __init__(self):
            self.torch = torch
            self.dt = float(dt)
            self.snes_rtol, self.snes_atol, self.snes_stol = 1e-12, 1e-50, 1e-14
            self.ksp_rtol, self.restart, self.max_newton, self.ksp_max_it = 1e-12, 30, 10, 1000
            self.stream = None
            self.jvp_mode, self.scale = 0, True
            self.owned = torch.cat([torch.ones(n, 1), torch.zeros(3, 1)]).double()
            self.prev = None
            self.stats = {"steps": 0, "newton": 0, "gmres": 0, "rhs": 0, "jvp": 0, "ksp_unconverged": 0, "snes_unconverged": 0}
            self.log = []
            self.reductions = []

        def _set_mode(self, mode):
            pass

        def _fill(self, U):
            U[n:] = U[:3]

        def _rhs(self, U):
            F = torch.zeros_like(U)
            F[:n] = (A @ U[:n].reshape(-1)).reshape(n, nc)
            return F

        def _fill_tangent(self, dU):
            dU[n:] = dU[:3]

        def _jvp(self, U, dU):
            return self._rhs(dU)

    return Fake()


def test_bdf_steps_match_the_dense_linear_solution():
    torch = pytest.importorskip("torch")
    p = _LinearProblem()
    dt = 0.05
    st = _stepper(p, dt, torch)
    rng = np.random.default_rng(5)
    U = torch.from_numpy(rng.standard_normal((p.n + 3, p.nc)))
    u0 = U[:p.n].reshape(-1).numpy().copy()
    st.step(U)
    st.step(U)
    I = np.eye(p.n * p.nc)
    u1 = np.linalg.solve(I - dt * p.A, u0)
    u2 = np.linalg.solve(I - 2 / 3 * dt * p.A, 4 / 3 * u1 - 1 / 3 * u0)
    np.testing.assert_allclose(U[:p.n].reshape(-1).numpy(), u2, rtol=0, atol=1e-10 * np.abs(u2).max())
    assert torch.equal(U[p.n:], U[:3])
    assert st.stats["steps"] == 2 and st.stats["snes_unconverged"] == 0 and st.stats["ksp_unconverged"] == 0
