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


@pytest.mark.parametrize("solver", [4, 2])
def test_torch_backend_matches_numpy(solver):
    """The torch float64 backend (the benchmark's FP64 gradient check on the
    GPU) is the numpy restatement operation for operation: loss and every
    gradient agree to 1e-12 (FFT libraries differ in the last bits)."""
    torch = pytest.importorskip("torch")  # noqa: F841
    prob, m0, th, _ = case(n=10, steps=16, solver=solver)
    loss, g = prob.backward(m0, th)
    p2 = R.Problem((10, 10, 1), CELL, 0.02, (1.0, 0.0, 0.0), 1e-13, 16, prob.probe, prob.avg_from,
                   target=prob.target, solver=solver, backend="torch", device="cpu")
    loss2, g2 = p2.backward(m0, th)
    assert loss2 == pytest.approx(loss, rel=1e-12)
    for k in ("A", "K1"):
        assert g2[k] == pytest.approx(g[k], rel=1e-10)
    for k in ("Ms", "B", "m0"):
        a, b = np.asarray(g2[k]), np.asarray(g[k])
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), k


def dmi_case(N=(10, 8, 1), steps=20, seed=6, solver=4, D=3e-3, Ku_axis=(0.0, 0.0, 1.0), pbc=(0, 0, 0)):
    """Exchange + interfacial DMI (the multilayer's material: D 3e-3 J/m^2,
    Ku1 along z), 2D or 3D, open or periodic."""
    rng = np.random.default_rng(seed)
    shape = (N[2], N[1], N[0])
    Ms = rng.uniform(9e5, 1.2e6, shape)
    m0 = rng.normal(size=(3,) + shape)
    t = rng.normal(size=3)
    t /= np.linalg.norm(t)
    prob = R.Problem(N, (2e-9, 2e-9, 1e-9), 0.3, Ku_axis, 5e-14, steps, (1, 1, N[0] // 2, N[1] // 2),
                     steps - steps // 4 + 1, target=t, solver=solver, Dind=D, pbc=pbc)
    th = R.params(Ms, 1.6e-11, 5e5, (0.0, 0.0, 0.05))
    return prob, m0, th, rng


def test_dmi_field_is_the_reference_restatement():
    """The FP64 dmi() equals the CPU oracle's dmi.cl restatement (orc_add_dmi,
    FP64) on a 3D mesh, and is its own transpose."""
    from oracle import oracle as O
    prob, m0, th, rng = dmi_case(N=(9, 7, 3))
    m = m0 / np.sqrt((m0 * m0).sum(0))
    B = np.zeros_like(m)
    A, D = th["A"], prob.D
    O.add_dmi(B, m, O.exch_lut(np.full(256, A), dtype=np.float64), O.exch_lut(np.full(256, D), dtype=np.float64),
              np.zeros(m.shape[1:], np.uint8), prob.cell, 1.0)
    h = prob.dmi(m, A)
    assert np.abs(h - B).max() <= 1e-13 * np.abs(B).max()
    x, y = rng.normal(size=m.shape), rng.normal(size=m.shape)
    lhs, rhs = (x * prob.dmi(y, A)).sum(), (prob.dmi(x, A) * y).sum()
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("N,solver", [((10, 8, 1), 4), ((8, 6, 3), 4), ((10, 8, 1), 2)])
def test_dmi_reverse_pass_matches_central_fd(N, solver):
    prob, m0, th, rng = dmi_case(N=N, solver=solver)
    _, g = prob.backward(m0, th)
    checks = [("A", None), ("K1", None), ("B", 0), ("B", 1), ("B", 2)]
    cells = rng.choice(N[0] * N[1] * N[2], size=24, replace=False)
    for c in cells:
        z, r = divmod(int(c), N[0] * N[1])
        checks.append(("Ms", (z, r // N[0], r % N[0])))
    for which in checks:
        fd = R.fd_gradient(prob, m0, th, which, rel=1e-4)
        ad = g[which[0]] if which[1] is None else g[which[0]][which[1]]
        assert abs(fd - ad) <= 1e-4 * abs(fd) + 1e-12 * max(1.0, abs(ad)), (which, fd, ad)


def test_periodic_dmi_field_is_the_reference_restatement():
    """With periodic x and y the FP64 dmi() equals the CPU oracle's dmi.cl
    restatement with wrapped neighbours (PBC code 3), and stays its own
    transpose; so does the periodic exchange stencil."""
    from oracle import oracle as O
    prob, m0, th, rng = dmi_case(N=(9, 7, 3), pbc=(2, 3, 0))
    m = m0 / np.sqrt((m0 * m0).sum(0))
    B = np.zeros_like(m)
    A, D = th["A"], prob.D
    O.add_dmi(B, m, O.exch_lut(np.full(256, A), dtype=np.float64), O.exch_lut(np.full(256, D), dtype=np.float64),
              np.zeros(m.shape[1:], np.uint8), prob.cell, 1.0, pbc=3)
    h = prob.dmi(m, A)
    assert np.abs(h - B).max() <= 1e-13 * np.abs(B).max()
    x, y = rng.normal(size=m.shape), rng.normal(size=m.shape)
    lhs, rhs = (x * prob.dmi(y, A)).sum(), (prob.dmi(x, A) * y).sum()
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    lhs, rhs = (x * prob.stencil(y)).sum(), (prob.stencil(x) * y).sum()
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("N,pbc,D", [((10, 8, 1), (2, 0, 0), 3e-3), ((8, 6, 3), (1, 1, 1), 3e-3),
                                     ((10, 8, 1), (0, 2, 0), 0.0)])
def test_periodic_reverse_pass_matches_central_fd(N, pbc, D):
    """Periodic meshes (the demag kernel's images, wrapped stencils): the
    reverse pass against central differences."""
    prob, m0, th, rng = dmi_case(N=N, pbc=pbc, D=D)
    _, g = prob.backward(m0, th)
    checks = [("A", None), ("K1", None), ("B", 0), ("B", 1), ("B", 2)]
    cells = rng.choice(N[0] * N[1] * N[2], size=16, replace=False)
    for c in cells:
        z, r = divmod(int(c), N[0] * N[1])
        checks.append(("Ms", (z, r // N[0], r % N[0])))
    for which in checks:
        fd = R.fd_gradient(prob, m0, th, which, rel=1e-4)
        ad = g[which[0]] if which[1] is None else g[which[0]][which[1]]
        assert abs(fd - ad) <= 1e-4 * abs(fd) + 1e-12 * max(1.0, abs(ad)), (which, fd, ad)


def _holes(N, seed=9):
    """A geometry with holes: a disc-like region plus a few empty cells
    inside it, and one partial-volume cell."""
    rng = np.random.default_rng(seed)
    Nx, Ny, Nz = N
    yy, xx = np.mgrid[0:Ny, 0:Nx]
    disc = (((xx - Nx / 2 + 0.5) / (Nx / 2)) ** 2 + ((yy - Ny / 2 + 0.5) / (Ny / 2)) ** 2 <= 1.0).astype(np.float64)
    g = np.repeat(disc[None], Nz, axis=0)
    inner = np.argwhere(g > 0)
    for z, y, x in inner[rng.choice(len(inner), size=3, replace=False)]:
        g[z, y, x] = 0.0
    z, y, x = inner[rng.choice(len(inner))]
    if g[z, y, x] > 0:
        g[z, y, x] = 0.6
    return g


@pytest.mark.parametrize("D", [3e-3, 0.0])
def test_geometry_operators_are_symmetric_and_restate_the_reference(D):
    """With a geometry the masked exchange stencil and the DMI field stay
    their own transposes, and the DMI field equals the CPU oracle's dmi.cl
    restatement on the masked state (a zero m is a missing neighbour)."""
    from oracle import oracle as O
    N = (9, 8, 3)
    g = _holes(N)
    prob, m0, th, rng = dmi_case(N=N, D=D if D else 3e-3)
    prob = R.Problem(N, prob.cell, 0.3, (0.0, 0.0, 1.0), 5e-14, 4, (1, 1, 2, 2), 3, Dind=D, geom=g)
    m = prob.normalize(m0)
    assert np.all(m[:, g == 0] == 0)
    x, y = rng.normal(size=m.shape) * (g > 0), rng.normal(size=m.shape) * (g > 0)
    A = th["A"]
    for op in ((lambda v: prob.dmi(v, A)) if D else None, prob.stencil):
        if op is None:
            continue
        lhs, rhs = (x * op(y)).sum(), (op(x) * y).sum()
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    if D:
        B = np.zeros_like(m)
        O.add_dmi(B, m, O.exch_lut(np.full(256, A), dtype=np.float64), O.exch_lut(np.full(256, D), dtype=np.float64),
                  np.zeros(m.shape[1:], np.uint8), prob.cell, 1.0)
        h = prob.dmi(m, A)
        assert np.abs(h - B * (g > 0)).max() <= 1e-13 * np.abs(B).max()


@pytest.mark.parametrize("N,D,solver", [((10, 8, 1), 3e-3, 4), ((8, 8, 2), 0.0, 4), ((10, 8, 1), 3e-3, 2)])
def test_geometry_reverse_pass_matches_central_fd(N, D, solver):
    """With a geometry (holes and a partial cell): the reverse pass against
    central differences."""
    g = _holes(N)
    prob0, m0, th, rng = dmi_case(N=N, solver=solver)
    prob = R.Problem(N, prob0.cell, 0.3, (0.0, 0.0, 1.0), 5e-14, 20, (1, 1, N[0] // 2, N[1] // 2), 16,
                     target=np.array([0.0, 0.6, 0.8]), solver=solver, Dind=D, geom=g)
    _, gr = prob.backward(m0, th)
    assert np.all(gr["Ms"][g == 0] == 0) and np.all(gr["m0"][:, g == 0] == 0)
    checks = [("A", None), ("K1", None), ("B", 0), ("B", 1), ("B", 2)]
    cells = np.argwhere(g > 0)
    for z, y, x in cells[rng.choice(len(cells), size=12, replace=False)]:
        checks.append(("Ms", (int(z), int(y), int(x))))
    for which in checks:
        fd = R.fd_gradient(prob, m0, th, which, rel=1e-4)
        ad = gr[which[0]] if which[1] is None else gr[which[0]][which[1]]
        assert abs(fd - ad) <= 1e-4 * abs(fd) + 1e-12 * max(1.0, abs(ad)), (which, fd, ad)


def region_case(N=(10, 8, 1), steps=16, seed=8, solver=4, geom=None, pbc=(0, 0, 0)):
    """Three regions (stripes along x and a block) with their own A, K1 and
    applied field."""
    rng = np.random.default_rng(seed)
    shape = (N[2], N[1], N[0])
    reg = np.zeros(shape, np.uint8)
    reg[:, :, N[0] // 3:] = 1
    reg[:, N[1] // 2:, 2 * N[0] // 3:] = 2
    Ms = rng.uniform(9e5, 1.2e6, shape)
    m0 = rng.normal(size=(3,) + shape)
    t = rng.normal(size=3)
    t /= np.linalg.norm(t)
    prob = R.Problem(N, (2e-9, 2e-9, 1e-9), 0.3, (0.0, 0.6, 0.8), 5e-14, steps, (1, 1, N[0] // 2, N[1] // 2),
                     steps - steps // 4 + 1, target=t, solver=solver, regions=reg, geom=geom, pbc=pbc)
    th = R.params(Ms, [1.6e-11, 0.9e-11, 1.3e-11], [5e5, 2e5, 0.0],
                  [(0.0, 0.0, 0.05), (0.02, 0.0, 0.03), (0.0, -0.01, 0.04)])
    return prob, m0, th, rng, reg


def test_one_region_equals_the_uniform_problem():
    """A region map with a single region gives the uniform problem's loss
    and gradients (per-region arrays of length one)."""
    N = (9, 7, 2)
    prob, m0, th, rng, reg = region_case(N=N)
    one = np.zeros_like(reg)
    pr = R.Problem(N, prob.cell, 0.3, (0.0, 0.6, 0.8), 5e-14, 16, prob.probe, prob.avg_from, target=prob.target,
                   regions=one)
    pu = R.Problem(N, prob.cell, 0.3, (0.0, 0.6, 0.8), 5e-14, 16, prob.probe, prob.avg_from, target=prob.target)
    thr = R.params(th["Ms"], [1.4e-11], [3e5], [(0.01, 0.0, 0.05)])
    thu = R.params(th["Ms"], 1.4e-11, 3e5, (0.01, 0.0, 0.05))
    lr, gr = pr.backward(m0, thr)
    lu, gu = pu.backward(m0, thu)
    assert abs(lr - lu) <= 1e-14 * abs(lu)
    assert abs(gr["A"][0] - gu["A"]) <= 1e-10 * abs(gu["A"])
    assert abs(gr["K1"][0] - gu["K1"]) <= 1e-10 * abs(gu["K1"])
    np.testing.assert_allclose(gr["B"][0], gu["B"], rtol=1e-10)
    np.testing.assert_allclose(gr["Ms"], gu["Ms"], rtol=1e-9, atol=1e-12 * np.abs(gu["Ms"]).max())


@pytest.mark.parametrize("N,geom,pbc", [((10, 8, 1), False, (0, 0, 0)), ((8, 8, 2), True, (0, 0, 0)),
                                        ((10, 8, 1), False, (2, 0, 0))])
def test_region_reverse_pass_matches_central_fd(N, geom, pbc):
    """Per-region A (pair coefficients the harmonic means), K1 and B_ext
    with a region map, on an open, masked or periodic mesh: the reverse
    pass against central differences."""
    g = _holes(N) if geom else None
    prob, m0, th, rng, reg = region_case(N=N, geom=g, pbc=pbc)
    _, gr = prob.backward(m0, th)
    checks = [("A", 0), ("A", 1), ("A", 2), ("K1", 0), ("K1", 1), ("B", (1, 0)), ("B", (2, 1)), ("B", (0, 2))]
    cells = np.argwhere(g > 0) if geom else np.argwhere(np.ones(reg.shape))
    for z, y, x in cells[rng.choice(len(cells), size=8, replace=False)]:
        checks.append(("Ms", (int(z), int(y), int(x))))
    for which in checks:
        fd = R.fd_gradient(prob, m0, th, which, rel=1e-4)
        ad = gr[which[0]][which[1]]
        assert abs(fd - ad) <= 1e-4 * abs(fd) + 1e-12 * max(1.0, abs(ad)), (which, fd, ad)
