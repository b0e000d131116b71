"""GPU adjoint (umag_adj_*): the forward pass against the engine's RK4 and Heun, the
gradients against the FP64 oracle's reverse pass (itself pinned to central
finite differences in tests/test_oracle_adjoint.py), and the autograd
wrapper.  The problem is the differentiation workload (per-cell Ms map in
[6e5, 9e5] A/m, Aex 1.3e-11 J/m, Ku1 2e5 J/m^3 along x, alpha 0.02,
B_ext (5, 5, 0) mT, fixed-step RK4 with dt 1e-13 s) on a smaller film and
fewer steps, so that the FP64 oracle finishes in seconds."""
import numpy as np
import pytest
import torch

from oracle import adjoint_ref as R

pytestmark = pytest.mark.gpu

CELL = (4e-9, 4e-9, 4e-9)
A_EX, KU1, BEXT = 1.3e-11, 2e5, (5e-3, 5e-3, 0.0)


def make_case(n, steps, seed):
    rng = np.random.default_rng(seed)
    Ms = rng.uniform(6e5, 9e5, (1, n, n)).astype(np.float32)
    m0 = rng.normal(size=(3, 1, n, n))
    m0 = (m0 / np.linalg.norm(m0, axis=0)).astype(np.float32)
    t = rng.normal(size=3)
    t /= np.linalg.norm(t)
    w = max(2, n // 8)
    kw = dict(N=(n, n, 1), cell=CELL, alpha=0.02, anisU=(1.0, 0.0, 0.0), dt=1e-13, nsteps=steps,
              probe=(n // 2 - w // 2, n // 2 - w // 2, w, w), avg_from=steps - steps // 4 + 1, target=tuple(t))
    return Ms, m0, kw


def gpu_sim(kw, K, use_graph=True, solver=4):
    from umagnus_b200.adjoint import AdjointRK4
    return AdjointRK4(K=K, use_graph=use_graph, solver=solver, **kw)


@pytest.mark.parametrize("solver", [4, 2])
def test_forward_matches_engine(solver):
    """The adjoint's forward pass is the engine's fixed-step RK4 (or Heun),
    bit for bit."""
    from umagnus_b200.engine import Simulation
    Ms, m0, kw = make_case(32, 40, 1)
    adj = gpu_sim(kw, K=16, solver=solver)
    adj.forward(m0, Ms, A_EX, KU1, BEXT)
    m_adj = adj.final_m().cpu().numpy()
    sim = Simulation(kw["N"], CELL, Msat=Ms, Aex=A_EX, alpha=0.02, Ku1=KU1, anisU=(1.0, 0.0, 0.0), B_ext=BEXT,
                     solver=solver, dt=1e-13, FixDt=1e-13)
    sim.set_m(m0)
    sim.steps(40)
    m_eng = sim.get_m().cpu().numpy().reshape(m_adj.shape)
    assert np.array_equal(m_adj, m_eng), np.abs(m_adj - m_eng).max()


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n,steps,K,solver", [(16, 30, 7, 4), (32, 60, 16, 4), (16, 30, 7, 2), (32, 60, 16, 2)])
def test_gradients_match_fp64_oracle(n, steps, K, solver):
    Ms, m0, kw = make_case(n, steps, 2 + n)
    adj = gpu_sim(kw, K=K, solver=solver)
    loss = adj.forward(m0, Ms, A_EX, KU1, BEXT)
    g = adj.backward()
    prob = R.Problem(solver=solver, **{k: v for k, v in kw.items()})
    th = R.params(Ms.astype(np.float64), A_EX, KU1, BEXT)
    loss64, g64 = prob.backward(m0.astype(np.float64), th)
    assert abs(loss - loss64) <= 1e-5 * max(1.0, abs(loss64))
    errs = {"Ms": _rel(g["Ms"].cpu().numpy(), g64["Ms"]), "m0": _rel(g["m0"].cpu().numpy(), g64["m0"]),
            "Aex": _rel(g["Aex"], g64["A"]), "Ku1": _rel(g["Ku1"], g64["K1"]),
            "B_ext": _rel(g["B_ext"], g64["B"])}
    print("relative gradient error vs FP64:", errs)
    for k, e in errs.items():
        assert e < 1e-3, (k, e)


def _run(kw, K, Ms, m0, use_graph=True, solver=4):
    adj = gpu_sim(kw, K=K, use_graph=use_graph, solver=solver)
    loss = adj.forward(m0, Ms, A_EX, KU1, BEXT)
    g = adj.backward()
    return (loss, g["Ms"].cpu().numpy(), g["m0"].cpu().numpy(), g["Aex"], g["Ku1"], tuple(g["B_ext"]))


def _same(a, b):
    assert a[0] == b[0]
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert a[3:] == b[3:]


@pytest.mark.parametrize("solver", [4, 2])
def test_segment_length_does_not_change_gradients(solver):
    """The checkpoint interval K only changes what is recomputed: results
    are bit-identical (per-cell FP64 accumulators, fixed-order reduction)."""
    Ms, m0, kw = make_case(16, 24, 9)
    ref = _run(kw, 24, Ms, m0, solver=solver)
    for K in (1, 5, 7):
        _same(_run(kw, K, Ms, m0, solver=solver), ref)


def test_graphs_match_stream_launches():
    Ms, m0, kw = make_case(16, 20, 13)
    _same(_run(kw, 6, Ms, m0, use_graph=True), _run(kw, 6, Ms, m0, use_graph=False))


def test_repeated_calls_and_new_parameters():
    """Graphs are keyed by the baked-in parameters: a second forward with a
    different Aex must not replay the first one's graphs."""
    Ms, m0, kw = make_case(16, 12, 17)
    adj = gpu_sim(kw, K=4)
    l1 = adj.forward(m0, Ms, A_EX, KU1, BEXT)
    l2 = adj.forward(m0, Ms, 2 * A_EX, KU1, BEXT)
    l3 = adj.forward(m0, Ms, A_EX, KU1, BEXT)
    fresh = gpu_sim(kw, K=4, use_graph=False)
    assert l1 == l3 and l2 == fresh.forward(m0, Ms, 2 * A_EX, KU1, BEXT) and l1 != l2


def test_autograd_function():
    Ms, m0, kw = make_case(16, 20, 11)
    adj = gpu_sim(kw, K=8)
    dev = torch.device("cuda", 0)
    tMs = torch.tensor(Ms, device=dev, requires_grad=True)
    tm0 = torch.tensor(m0, device=dev, requires_grad=True)
    tA = torch.tensor(A_EX, dtype=torch.float64, requires_grad=True)
    tK = torch.tensor(KU1, dtype=torch.float64, requires_grad=True)
    tB = torch.tensor(BEXT, dtype=torch.float64, requires_grad=True)
    loss = adj.loss(tm0, tMs, tA, tK, tB)
    (2.0 * loss).backward()
    ref = gpu_sim(kw, K=8)
    ref.forward(m0, Ms, A_EX, KU1, BEXT)
    g = ref.backward()
    assert torch.equal(tMs.grad, 2.0 * g["Ms"])
    assert torch.equal(tm0.grad, 2.0 * g["m0"])
    assert float(tA.grad) == 2.0 * g["Aex"]
    assert float(tK.grad) == 2.0 * g["Ku1"]
    assert np.allclose(tB.grad.numpy(), 2.0 * np.asarray(g["B_ext"]), rtol=0, atol=0)


def test_argument_errors():
    from umagnus_b200._lib import UmagError
    Ms, m0, kw = make_case(16, 10, 3)
    bad = dict(kw, avg_from=11)
    with pytest.raises(UmagError):
        gpu_sim(bad, K=4)
    bad = dict(kw, probe=(10, 10, 8, 8))
    with pytest.raises(UmagError):
        gpu_sim(bad, K=4)
    adj = gpu_sim(kw, K=4)
    with pytest.raises(UmagError):
        adj.backward()  # no forward yet
    with pytest.raises(UmagError):
        gpu_sim(kw, K=4, solver=5)  # RK4 and Heun only


# ---------------------------------------------------------------- interfacial DMI
MULTI = dict(cell=(2e-9, 2e-9, 1e-9), alpha=0.3, anisU=(0.0, 0.0, 1.0), dt=5e-14)
M_AEX, M_KU1, M_BEXT, M_D = 1.6e-11, 5e5, (0.0, 0.0, 0.05), 3e-3


def multilayer_case(N, steps, seed):
    """The multilayer's material (Aex 1.6e-11, D 3e-3, Ku1 5e5 along z,
    alpha 0.3, B_ext (0, 0, 50 mT), 2x2x1 nm cells) on a small mesh with a
    per-cell Ms map around 1.1e6 A/m."""
    rng = np.random.default_rng(seed)
    shape = (N[2], N[1], N[0])
    Ms = rng.uniform(1.0e6, 1.2e6, shape).astype(np.float32)
    m0 = rng.normal(size=(3,) + shape)
    m0 = (m0 / np.linalg.norm(m0, axis=0)).astype(np.float32)
    t = rng.normal(size=3)
    t /= np.linalg.norm(t)
    kw = dict(N=N, nsteps=steps, probe=(2, 2, N[0] // 2, N[1] // 2), avg_from=steps - steps // 4 + 1,
              target=tuple(t), **MULTI)
    return Ms, m0, kw


@pytest.mark.parametrize("solver", [4, 2])
def test_dmi_forward_matches_engine(solver):
    """With interfacial DMI on a 3D mesh the adjoint's forward is still the
    engine's fixed-step stepper bit for bit (dmi.cl arithmetic)."""
    from umagnus_b200.engine import Simulation
    Ms, m0, kw = multilayer_case((16, 12, 3), 24, 5)
    adj = gpu_sim(dict(kw, Dind=M_D), K=8, solver=solver)
    adj.forward(m0, Ms, M_AEX, M_KU1, M_BEXT)
    m_adj = adj.final_m().cpu().numpy()
    sim = Simulation(kw["N"], kw["cell"], Msat=Ms, Aex=M_AEX, alpha=kw["alpha"], Dind=M_D, Ku1=M_KU1,
                     anisU=kw["anisU"], B_ext=M_BEXT, solver=solver, dt=kw["dt"], FixDt=kw["dt"])
    sim.set_m(m0)
    sim.steps(24)
    m_eng = sim.get_m().cpu().numpy().reshape(m_adj.shape)
    assert np.array_equal(m_adj, m_eng), np.abs(m_adj - m_eng).max()


@pytest.mark.parametrize("N,solver", [((24, 16, 1), 4), ((16, 12, 4), 4), ((16, 12, 4), 2)])
def test_dmi_gradients_match_fp64_oracle(N, solver):
    """Gradients through the transposed DMI stencil (including the
    extrapolated boundary neighbours) against the FP64 reverse pass, which
    tests/test_oracle_adjoint.py pins to central differences."""
    Ms, m0, kw = multilayer_case(N, 30, 7 + N[2])
    adj = gpu_sim(dict(kw, Dind=M_D), K=8, solver=solver)
    loss = adj.forward(m0, Ms, M_AEX, M_KU1, M_BEXT)
    g = adj.backward()
    prob = R.Problem(solver=solver, Dind=M_D, **kw)
    th = R.params(Ms.astype(np.float64), M_AEX, M_KU1, M_BEXT)
    loss64, g64 = prob.backward(m0.astype(np.float64), th)
    assert abs(loss - loss64) <= 1e-5 * max(1.0, abs(loss64))
    errs = {"Ms": _rel(g["Ms"].cpu().numpy(), g64["Ms"]), "m0": _rel(g["m0"].cpu().numpy(), g64["m0"]),
            "Aex": _rel(g["Aex"], g64["A"]), "Ku1": _rel(g["Ku1"], g64["K1"]),
            "B_ext": _rel(g["B_ext"], g64["B"])}
    print("relative gradient error vs FP64 (DMI):", errs)
    for k, e in errs.items():
        assert e < 1e-3, (k, e)


# ---------------------------------------------------------------- periodic meshes
@pytest.mark.parametrize("N,pbc,dmi", [((16, 12, 1), (2, 0, 0), True), ((16, 12, 4), (1, 1, 0), True),
                                       ((16, 12, 3), (0, 2, 1), False)])
def test_periodic_forward_matches_engine(N, pbc, dmi):
    """On a periodic mesh (the demag kernel's images, wrapped stencils) the
    adjoint's forward is the engine's fixed-step RK4 with the same PBC, bit
    for bit."""
    from umagnus_b200.engine import Simulation
    Ms, m0, kw = multilayer_case(N, 24, 11 + N[2])
    D = M_D if dmi else 0.0
    adj = gpu_sim(dict(kw, Dind=D, pbc=pbc), K=8)
    adj.forward(m0, Ms, M_AEX, M_KU1, M_BEXT)
    m_adj = adj.final_m().cpu().numpy()
    sim = Simulation(kw["N"], kw["cell"], Msat=Ms, Aex=M_AEX, alpha=kw["alpha"], Dind=D, Ku1=M_KU1,
                     anisU=kw["anisU"], B_ext=M_BEXT, solver=4, dt=kw["dt"], FixDt=kw["dt"], pbc=pbc)
    sim.set_m(m0)
    sim.steps(24)
    m_eng = sim.get_m().cpu().numpy().reshape(m_adj.shape)
    assert np.array_equal(m_adj, m_eng), np.abs(m_adj - m_eng).max()


@pytest.mark.parametrize("N,pbc,dmi", [((16, 12, 1), (2, 0, 0), True), ((16, 12, 4), (1, 1, 1), True),
                                       ((24, 16, 1), (0, 3, 0), False)])
def test_periodic_gradients_match_fp64_oracle(N, pbc, dmi):
    """Gradients on periodic meshes against the FP64 reverse pass with the
    same PBC (pinned to central differences in tests/test_oracle_adjoint.py)."""
    Ms, m0, kw = multilayer_case(N, 30, 5 + N[2])
    D = M_D if dmi else 0.0
    adj = gpu_sim(dict(kw, Dind=D, pbc=pbc), K=8)
    loss = adj.forward(m0, Ms, M_AEX, M_KU1, M_BEXT)
    g = adj.backward()
    prob = R.Problem(Dind=D, pbc=pbc, **kw)
    th = R.params(Ms.astype(np.float64), M_AEX, M_KU1, M_BEXT)
    loss64, g64 = prob.backward(m0.astype(np.float64), th)
    assert abs(loss - loss64) <= 1e-5 * max(1.0, abs(loss64))
    errs = {"Ms": _rel(g["Ms"].cpu().numpy(), g64["Ms"]), "m0": _rel(g["m0"].cpu().numpy(), g64["m0"]),
            "Aex": _rel(g["Aex"], g64["A"]), "Ku1": _rel(g["Ku1"], g64["K1"]),
            "B_ext": _rel(g["B_ext"], g64["B"])}
    print("relative gradient error vs FP64 (periodic):", errs)
    for k, e in errs.items():
        assert e < 1e-3, (k, e)


# ---------------------------------------------------------------- geometry
def _geometry(N, seed=3):
    """A disc per layer with three empty cells inside and one cell of
    volume fraction 0.6."""
    rng = np.random.default_rng(seed)
    Nx, Ny, Nz = N
    yy, xx = np.mgrid[0:Ny, 0:Nx]
    disc = (((xx - Nx / 2 + 0.5) / (Nx / 2)) ** 2 + ((yy - Ny / 2 + 0.5) / (Ny / 2)) ** 2 <= 1.0).astype(np.float32)
    g = np.repeat(disc[None], Nz, axis=0)
    inner = np.argwhere(g > 0)
    pick = inner[rng.choice(len(inner), size=4, replace=False)]
    for z, y, x in pick[:3]:
        g[z, y, x] = 0.0
    z, y, x = pick[3]
    g[z, y, x] = 0.6
    return g


@pytest.mark.parametrize("N,dmi,solver", [((16, 12, 1), True, 4), ((16, 12, 3), False, 4), ((16, 12, 1), True, 2)])
def test_geometry_forward_matches_engine(N, dmi, solver):
    """With a geometry (holes, a partial cell) the adjoint's forward is the
    engine's fixed-step run with the same geometry, bit for bit."""
    from umagnus_b200.engine import Simulation
    Ms, m0, kw = multilayer_case(N, 24, 21 + N[2])
    g = _geometry(N)
    D = M_D if dmi else 0.0
    adj = gpu_sim(dict(kw, Dind=D, geom=g), K=8, solver=solver)
    adj.forward(m0, Ms, M_AEX, M_KU1, M_BEXT)
    m_adj = adj.final_m().cpu().numpy()
    sim = Simulation(kw["N"], kw["cell"], Msat=Ms, Aex=M_AEX, alpha=kw["alpha"], Dind=D, Ku1=M_KU1,
                     anisU=kw["anisU"], B_ext=M_BEXT, solver=solver, dt=kw["dt"], FixDt=kw["dt"], geom=g)
    sim.set_m(m0)
    sim.steps(24)
    m_eng = sim.get_m().cpu().numpy().reshape(m_adj.shape)
    assert np.array_equal(m_adj, m_eng), np.abs(m_adj - m_eng).max()
    assert np.all(m_adj.reshape(3, -1)[:, g.ravel() == 0] == 0)


@pytest.mark.parametrize("N,dmi,solver", [((16, 12, 1), True, 4), ((16, 12, 3), False, 4), ((16, 12, 2), True, 2)])
def test_geometry_gradients_match_fp64_oracle(N, dmi, solver):
    """Gradients with a geometry against the FP64 reverse pass with the same
    geometry (pinned to central differences in tests/test_oracle_adjoint.py);
    cells outside the geometry get zero Ms and m0 gradients."""
    Ms, m0, kw = multilayer_case(N, 30, 13 + N[2])
    g = _geometry(N)
    D = M_D if dmi else 0.0
    adj = gpu_sim(dict(kw, Dind=D, geom=g), K=8, solver=solver)
    loss = adj.forward(m0, Ms, M_AEX, M_KU1, M_BEXT)
    gr = adj.backward()
    prob = R.Problem(solver=solver, Dind=D, geom=g, **kw)
    th = R.params(Ms.astype(np.float64), M_AEX, M_KU1, M_BEXT)
    loss64, g64 = prob.backward(m0.astype(np.float64), th)
    assert abs(loss - loss64) <= 1e-5 * max(1.0, abs(loss64))
    gms = gr["Ms"].cpu().numpy().reshape(g.shape)
    assert np.all(gms[g == 0] == 0)
    assert np.all(gr["m0"].cpu().numpy().reshape((3,) + g.shape)[:, g == 0] == 0)
    errs = {"Ms": _rel(gms, g64["Ms"]), "m0": _rel(gr["m0"].cpu().numpy(), g64["m0"]),
            "Aex": _rel(gr["Aex"], g64["A"]), "Ku1": _rel(gr["Ku1"], g64["K1"]),
            "B_ext": _rel(gr["B_ext"], g64["B"])}
    print("relative gradient error vs FP64 (geometry):", errs)
    for k, e in errs.items():
        assert e < 1e-3, (k, e)


# ---------------------------------------------------------------- region maps
R_A, R_K1 = [1.6e-11, 0.9e-11, 1.3e-11], [5e5, 2e5, 0.0]
R_B = [(0.0, 0.0, 0.05), (0.02, 0.0, 0.03), (0.0, -0.01, 0.04)]


def _regions(N):
    reg = np.zeros(N[::-1], np.uint8)
    reg[:, :, N[0] // 3:] = 1
    reg[:, N[1] // 2:, 2 * N[0] // 3:] = 2
    return reg


@pytest.mark.parametrize("N,solver,geom", [((16, 12, 1), 4, False), ((16, 12, 3), 2, False), ((16, 12, 1), 4, True)])
def test_region_forward_matches_engine(N, solver, geom):
    """With a region map (per-region Aex through the engine's harmonic-mean
    LUT, per-region Ku1 and applied field) the adjoint's forward is the
    engine's fixed-step run of the same material, bit for bit."""
    from umagnus_b200.engine import Simulation
    Ms, m0, kw = multilayer_case(N, 24, 31 + N[2])
    reg = _regions(N)
    g = _geometry(N) if geom else None
    adj = gpu_sim(dict(kw, regions=reg, geom=g), K=8, solver=solver)
    adj.forward(m0, Ms, R_A, R_K1, R_B)
    m_adj = adj.final_m().cpu().numpy()
    bext = np.zeros((256, 3), np.float32)
    bext[:3] = R_B
    sim = Simulation(kw["N"], kw["cell"], Msat=Ms, Aex=R_A, alpha=kw["alpha"],
                     Ku1=np.asarray(R_K1, np.float32)[reg], anisU=kw["anisU"], B_ext=bext, regions=reg,
                     solver=solver, dt=kw["dt"], FixDt=kw["dt"], geom=g)
    sim.set_m(m0)
    sim.steps(24)
    m_eng = sim.get_m().cpu().numpy().reshape(m_adj.shape)
    assert np.array_equal(m_adj, m_eng), np.abs(m_adj - m_eng).max()


@pytest.mark.parametrize("N,solver,geom,pbc", [((16, 12, 1), 4, False, (0, 0, 0)), ((16, 12, 3), 4, True, (0, 0, 0)),
                                               ((16, 12, 1), 2, False, (2, 0, 0))])
def test_region_gradients_match_fp64_oracle(N, solver, geom, pbc):
    """Per-region gradients (Aex through the pair coefficients, Ku1, B_ext)
    and the Ms and m0 gradients against the FP64 reverse pass with the same
    region map (pinned to central differences in tests/test_oracle_adjoint.py)."""
    Ms, m0, kw = multilayer_case(N, 30, 41 + N[2])
    reg = _regions(N)
    g = _geometry(N) if geom else None
    adj = gpu_sim(dict(kw, regions=reg, geom=g, pbc=pbc), K=8, solver=solver)
    loss = adj.forward(m0, Ms, R_A, R_K1, R_B)
    gr = adj.backward()
    prob = R.Problem(solver=solver, regions=reg, geom=g, pbc=pbc, **kw)
    th = R.params(Ms.astype(np.float64), R_A, R_K1, R_B)
    loss64, g64 = prob.backward(m0.astype(np.float64), th)
    assert abs(loss - loss64) <= 1e-5 * max(1.0, abs(loss64))
    errs = {"Ms": _rel(gr["Ms"].cpu().numpy().reshape(reg.shape), g64["Ms"]),
            "m0": _rel(gr["m0"].cpu().numpy(), g64["m0"]),
            "Aex": _rel(gr["Aex"], g64["A"]), "Ku1": _rel(gr["Ku1"][:2], g64["K1"][:2]),
            "B_ext": _rel(gr["B_ext"], g64["B"])}
    print("relative gradient error vs FP64 (regions):", errs)
    for k, e in errs.items():
        assert e < 1e-3, (k, e)
    # every region's Aex gradient on its own, too
    for r in range(3):
        assert abs(gr["Aex"][r] - g64["A"][r]) <= 1e-3 * np.abs(g64["A"]).max(), (r, gr["Aex"], g64["A"])


def test_region_autograd_wrapper():
    """The torch.autograd form with per-region tensors."""
    from umagnus_b200.adjoint import AdjointRK4
    N = (16, 12, 1)
    Ms, m0, kw = multilayer_case(N, 12, 51)
    reg = _regions(N)
    adj = AdjointRK4(K=4, regions=reg, **kw)
    A = torch.tensor(R_A, dtype=torch.float64, requires_grad=True)
    K = torch.tensor(R_K1, dtype=torch.float64, requires_grad=True)
    B = torch.tensor(R_B, dtype=torch.float64, requires_grad=True)
    Mst = torch.tensor(Ms, requires_grad=True)
    loss = adj.loss(torch.tensor(m0), Mst, A, K, B)
    loss.backward()
    g = adj.backward()
    np.testing.assert_allclose(A.grad.numpy(), g["Aex"], rtol=1e-12)
    np.testing.assert_allclose(B.grad.numpy(), g["B_ext"], rtol=1e-12)
    assert A.grad.shape == (3,) and B.grad.shape == (3, 3) and Mst.grad.shape == Mst.shape
