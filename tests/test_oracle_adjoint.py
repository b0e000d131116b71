"""The FP64 oracle of the differentiable RK4 and Heun simulations: its reverse pass
against central finite differences of its own forward (relative step 1e-4,
randomly chosen cells), and the loss definition on hand-checkable cases.
CPU only."""
import numpy as np
import pytest

from oracle import adjoint_ref as R

CELL = (4e-9, 4e-9, 4e-9)


def case(n=12, steps=24, seed=5, demag=True, solver=4):
    rng = np.random.default_rng(seed)
    Ms = rng.uniform(6e5, 9e5, (1, n, n))
    m0 = rng.normal(size=(3, 1, n, n))
    t = rng.normal(size=3)
    t /= np.linalg.norm(t)
    prob = R.Problem((n, n, 1), CELL, 0.02, (1.0, 0.0, 0.0), 1e-13, steps, (n // 4, n // 4, n // 2, n // 2),
                     steps - steps // 4 + 1, target=t, demag=demag, solver=solver)
    th = R.params(Ms, 1.3e-11, 2e5, (5e-3, 5e-3, 0.0))
    return prob, m0, th, rng


@pytest.mark.parametrize("demag,solver", [(True, 4), (False, 4), (True, 2), (False, 2)])
def test_reverse_pass_matches_central_fd(demag, solver):
    prob, m0, th, rng = case(demag=demag, solver=solver)
    _, g = prob.backward(m0, th)
    checks = [("A", None), ("K1", None), ("B", 0), ("B", 1), ("B", 2)]
    n = m0.shape[-1]
    cells = rng.choice(n * n, size=64 if demag else 16, replace=False)
    checks += [("Ms", (0, int(c) // n, int(c) % n)) for c in cells]
    for which in checks:
        fd = R.fd_gradient(prob, m0, th, which, rel=1e-4)
        ad = g[which[0]] if which[1] is None else g[which[0]][which[1]]
        assert abs(fd - ad) <= 1e-4 * abs(fd) + 1e-12 * max(1.0, abs(ad)), (which, fd, ad)


@pytest.mark.parametrize("solver", [4, 2])
def test_m0_gradient_matches_fd(solver):
    prob, m0, th, rng = case(n=8, steps=12, solver=solver)
    _, g = prob.backward(m0, th)
    for _ in range(6):
        c, y, x = int(rng.integers(3)), int(rng.integers(8)), int(rng.integers(8))
        d = 1e-6
        mp, mm = m0.copy(), m0.copy()
        mp[c, 0, y, x] += d
        mm[c, 0, y, x] -= d
        fd = (prob.forward(mp, th) - prob.forward(mm, th)) / (2 * d)
        assert abs(fd - g["m0"][c, 0, y, x]) <= 1e-5 * abs(fd) + 1e-9, (fd, g["m0"][c, 0, y, x])


def test_loss_of_a_static_state():
    """A uniform state along z with no torque stays put: probe mean 1, and
    the target term is |(0,0,1) - target|^2."""
    n = 8
    prob = R.Problem((n, n, 1), CELL, 0.1, (0.0, 0.0, 1.0), 1e-13, 5, (0, 0, 4, 4), 3, w_probe=2.0, w_target=3.0,
                     target=(1.0, 0.0, 0.0), demag=False)
    m0 = np.zeros((3, 1, n, n))
    m0[2] = 1.0
    th = R.params(np.full((1, n, n), 8e5), 1.3e-11, 0.0, (0.0, 0.0, 0.1))
    assert prob.forward(m0, th) == pytest.approx(2.0 * 1.0 + 3.0 * 2.0, abs=1e-12)
