"""Whole-step parity of the device engine (umag_sim_*) with the oracle.

Levels (the FFT rounding differs, so trajectories are compared at three
levels):  (1) one torque evaluation on identical m, |d tau| <= 1e-5 max|tau|;
(2) fixed-dt steps of every solver, max |dm| <= 1e-5 after a few steps;
(3) adaptive RK45DP runs: average m and accepted-step counts close to the
oracle's, and the error against the FP64 oracle reported.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_pins as G

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MU0 = G.MU0


@pytest.fixture(scope="module")
def eng():
    from umagnus_b200 import engine
    return engine


def thin_film(dtype=np.float32, **kw):
    """64x64x1 cells of 4x4x3 nm, Ms 8e5, Aex 1.3e-11, alpha 0.1, B=(0,0,10 mT)."""
    p = dict(N=(64, 64, 1), cell=(4e-9, 4e-9, 3e-9), Ms=8e5, Aex=1.3e-11, alpha=0.1, B_ext=(0, 0, 0.01))
    p.update(kw)
    return p


def multilayer_small(**kw):
    """The 3D multilayer material (DMI + anisotropy) on a smaller grid."""
    p = dict(N=(48, 40, 8), cell=(2e-9, 2e-9, 1e-9), Ms=1.1e6, Aex=1.6e-11, alpha=0.3, Dind=3e-3, Ku1=5e5,
             anisU=(0, 0, 1), B_ext=(0, 0, 0.05))
    p.update(kw)
    return p


def make_pair(eng, p, solver=5, fix_dt=0.0, seed=1):
    g = eng.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], Dind=p.get("Dind", 0.0),
                       Ku1=p.get("Ku1", 0.0), anisU=p.get("anisU", (0, 0, 1)), B_ext=p.get("B_ext"),
                       solver=solver, FixDt=fix_dt)
    o = O.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], Dind=p.get("Dind", 0.0),
                     Ku1=p.get("Ku1", 0.0), anisU=p.get("anisU", (0, 0, 1)), B_ext=p.get("B_ext"), solver=solver)
    o.solver.fix_dt = fix_dt
    m = G.random_unit(p["N"], seed)
    g.set_m(m)
    o.set_m(m)
    return g, o


@pytest.mark.parametrize("p", [thin_film(), multilayer_small()], ids=["film", "multilayer"])
def test_torque_matches_oracle(eng, p):
    g, o = make_pair(eng, p)
    # identical m on both sides (the device normalises in float32 exactly like the oracle)
    assert np.array_equal(g.get_m().cpu().numpy(), o.m)
    t, b = g.torque(beff=True)
    to, bo = o.torque(beff=True)
    t, b = t.cpu().numpy(), b.cpu().numpy()
    assert np.abs(b - bo).max() <= 1e-5 * np.abs(bo).max()
    assert np.abs(t - to).max() <= 1e-5 * np.abs(to).max()
    g.free()


def test_local_terms_bitexact_without_demag(eng):
    """With demag off every term is per-cell arithmetic: bit-identical to the oracle."""
    p = multilayer_small()
    g = eng.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], Dind=p["Dind"], Ku1=p["Ku1"],
                       anisU=p["anisU"], B_ext=p["B_ext"], demag=False)
    o = O.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], Dind=p["Dind"], Ku1=p["Ku1"],
                     anisU=p["anisU"], B_ext=p["B_ext"], demag=False)
    m = G.random_unit(p["N"], 4)
    g.set_m(m)
    o.set_m(m)
    t, b = g.torque(beff=True)
    to, bo = o.torque(beff=True)
    assert np.array_equal(b.cpu().numpy(), bo)
    assert np.array_equal(t.cpu().numpy(), to)
    g.free()


@pytest.mark.parametrize("case", ["cubic_uniform", "cubic_map_bulk_dmi", "bulk_dmi_regions"])
def test_cubic_and_bulk_dmi_bitexact_without_demag(eng, case):
    """Cubic anisotropy (engine/anisotropy.go:54-74) and bulk DMI
    (engine/exchange.go:60-61) in the engine's torque: bit-identical to the
    oracle, whose kernels are bit-identical to the reference's."""
    N, cell = (20, 14, 4), (2e-9, 2.5e-9, 1.5e-9)
    rng = np.random.default_rng(12)
    shape = (N[2], N[1], N[0])
    kw = dict(Ku1=2e5, anisU=(0.3, 0.1, 1.0), B_ext=(0.01, -0.02, 0.05))
    if case == "cubic_uniform":
        kw.update(Kc1=4.5e4, Kc2=-1.2e4, Kc3=3e3, anisC1=(1.0, 0.2, 0.0), anisC2=(-0.2, 1.0, 0.1))
    elif case == "cubic_map_bulk_dmi":
        kw.update(Kc1=(rng.random(shape) * 5e4).astype(np.float32), Kc2=2e4,
                  anisC1=rng.standard_normal((3,) + shape).astype(np.float32), anisC2=(0.0, 1.0, 0.0),
                  Dbulk=1.5e-3)
    else:
        kw.update(Dbulk=[2e-3, -1e-3], regions=rng.integers(0, 2, size=shape).astype(np.uint8))
    okw = dict(kw)
    if "regions" in kw and not np.isscalar(kw["Dbulk"]):
        dbk = np.zeros(256)
        dbk[:2] = kw["Dbulk"]
        okw.pop("Dbulk")
        okw["Dbulk_regions"] = dbk
    g = eng.Simulation(N, cell, 9e5, 1.2e-11, 0.1, demag=False, **kw)
    o = O.Simulation(N, cell, 9e5, 1.2e-11, 0.1, demag=False, **okw)
    m = G.random_unit(N, 5)
    g.set_m(m)
    o.set_m(m)
    t, b = g.torque(beff=True)
    to, bo = o.torque(beff=True)
    assert np.array_equal(b.cpu().numpy(), bo)
    assert np.array_equal(t.cpu().numpy(), to)
    E = g.energies()
    Eo = O.energies(o, o.m)
    scale = sum(abs(Eo[k]) for k in ("exchange", "anisotropy", "zeeman"))
    for k in ("exchange", "anisotropy", "zeeman", "total"):
        assert abs(E[k] - Eo[k]) <= 1e-5 * scale, (k, E[k], Eo[k])
    V = cell[0] * cell[1] * cell[2]
    assert float(g.energy_density().double().sum()) * V == pytest.approx(E["total"], rel=1e-5, abs=1e-9 * scale)
    g.free()


def test_interfacial_and_bulk_dmi_are_exclusive(eng):
    from umagnus_b200._lib import UmagError
    with pytest.raises(UmagError):
        eng.Simulation((8, 8, 1), (2e-9, 2e-9, 2e-9), 8e5, 1e-11, 0.1, Dind=1e-3, Dbulk=1e-3)


@pytest.mark.parametrize("solver", [1, 2, 3, 4, 5])
def test_fixed_step_trajectory(eng, solver):
    p = thin_film()
    g, o = make_pair(eng, p, solver=solver, fix_dt=2e-13)
    for _ in range(5):
        o.step()
    g.steps(5)
    st = g.state()
    assert st["nsteps"] == o.solver.nsteps == 5
    assert st["nevals"] == o.solver.nevals
    assert abs(st["time"] - o.solver.time) <= 1e-24
    dm = np.abs(g.get_m().cpu().numpy() - o.m).max()
    assert dm <= 1e-5
    g.free()


def test_adaptive_euler_steps(eng):
    """engine/euler.go:16-35 without FixDt: dt = MaxErr / max|torque| (a
    float32 step in units of GammaLL), every step accepted, LastErr = MaxErr
    up to the float32 rounding of dt."""
    p = thin_film()
    g, o = make_pair(eng, p, solver=1)
    for _ in range(6):
        o.step()
    g.steps(6)
    st = g.state()
    assert st["status"] == 0 and st["nsteps"] == o.solver.nsteps == 6 and st["nundone"] == 0
    assert st["nevals"] == o.solver.nevals == 6
    # dt follows max |torque|, whose last bits depend on the demag FFT rounding
    assert abs(st["time"] - o.solver.time) <= 1e-5 * o.solver.time
    assert abs(st["last_err"] - 1e-5) <= 1e-12
    assert abs(st["last_torque"] - o.solver.last_torque) <= 1e-5 * o.solver.last_torque
    assert np.abs(g.get_m().cpu().numpy() - o.m).max() <= 1e-5
    g.free()


def test_reassign_solver_and_alpha_between_runs(eng):
    """SetSolver / FixDt / alpha assigned between runs, as test/rk4.mx3 and
    test/euler.mx3 do: RK4 adaptive, then RK4 with FixDt and a new alpha,
    then Euler with FixDt, then RK4 adaptive again -- the oracle does the same."""
    p = thin_film(N=(32, 32, 1), alpha=0.5)
    g, o = make_pair(eng, p, solver=4)
    g.run(2e-12)
    o.run(2e-12)
    g.set_solver(FixDt=1e-13)
    g.set_param("alpha", 0.02)
    o.solver.fix_dt, o.sys.alpha_mul = 1e-13, float(np.float32(0.02))
    g.run(1e-12)
    o.run(1e-12)
    g.set_solver(1)
    o.solver.solver = 1
    g.run(5e-13)
    o.run(5e-13)
    g.set_solver(4, FixDt=0.0)
    o.solver.solver, o.solver.fix_dt = 4, 0.0
    g.run(1e-12)
    o.run(1e-12)
    st = g.state()
    assert st["status"] == 0
    assert abs(st["time"] - o.solver.time) <= 1e-22
    assert abs(st["nsteps"] - o.solver.nsteps) <= 2
    assert np.abs(g.get_m().cpu().numpy() - o.m).max() <= 1e-4
    g.free()


def test_set_param_matches_a_fresh_simulation(eng):
    """Msat, alpha, Ku1 reassigned on a running simulation give the torque a
    simulation created with those values gives, bit for bit."""
    p = multilayer_small()
    g, _ = make_pair(eng, p)
    g.steps(3)
    m = g.get_m().clone()
    rng = np.random.default_rng(5)
    shape = (p["N"][2], p["N"][1], p["N"][0])
    ku1 = (4e5 + 2e5 * rng.random(shape)).astype(np.float32)
    alpha = (0.1 + 0.2 * rng.random(shape)).astype(np.float32)
    g.set_param("Msat", 9.5e5)
    g.set_param("Ku1", ku1)
    g.set_param("alpha", alpha)
    f = eng.Simulation(p["N"], p["cell"], 9.5e5, p["Aex"], alpha, Dind=p["Dind"], Ku1=ku1, anisU=p["anisU"],
                       B_ext=p["B_ext"])
    f.set_m(m)
    g.set_m(m)
    tg, bg = g.torque(beff=True)
    tf, bf = f.torque(beff=True)
    assert torch.equal(bg, bf) and torch.equal(tg, tf)
    # and the next steps agree too (the step graphs were rebuilt)
    g.set_time(0.0, 5e-14)
    f.set_time(0.0, 5e-14)
    g.steps(4)
    f.steps(4)
    assert torch.equal(g.get_m(), f.get_m())
    with pytest.raises(Exception):
        g.set_param("Aex", 1.0)
    g.free()
    f.free()


def test_adaptive_rk45dp_short_run(eng):
    p = thin_film()
    g, o = make_pair(eng, p)
    g.run(2e-11)
    o.run(2e-11)
    st = g.state()
    assert st["status"] == 0
    assert abs(st["time"] - 2e-11) < 1e-22 and abs(o.solver.time - 2e-11) < 1e-22
    # accepted-step counts may differ by a few when a reject decision flips
    assert abs(st["nsteps"] - o.solver.nsteps) <= max(2, 0.05 * o.solver.nsteps)
    avg = np.array(g.average_m())
    avg_o = o.m.reshape(3, -1).astype(np.float64).mean(axis=1)
    assert np.abs(avg - avg_o).max() <= 1e-4
    g.free()


def test_graph_and_stream_paths_agree(eng):
    p = thin_film(N=(32, 32, 1))
    a, _ = make_pair(eng, p, fix_dt=1e-13)
    b, _ = make_pair(eng, p, fix_dt=1e-13)
    a.use_graph(True, 8)
    b.use_graph(False)
    a.steps(16)
    b.steps(16)
    assert torch.equal(a.get_m(), b.get_m())
    assert a.state()["nsteps"] == b.state()["nsteps"] == 16
    a.free()
    b.free()


def test_run_stops_exactly_at_alarm(eng):
    p = thin_film(N=(32, 32, 1))
    g, _ = make_pair(eng, p)
    g.run(1e-12, chunk=7)
    assert g.state()["time"] == pytest.approx(1e-12, rel=0, abs=1e-24)
    g.run(5e-13, chunk=3)
    assert g.state()["time"] == pytest.approx(1.5e-12, rel=0, abs=1e-24)
    g.free()


def test_frozen_spins(eng):
    """engine/torque.go:348-352 FreezeSpins: the torque is zero in frozen
    regions and unchanged elsewhere; frozen cells keep their m through steps."""
    p = multilayer_small(N=(24, 20, 4))
    regions = (np.arange(p["N"][0])[None, None, :] >= p["N"][0] // 2).astype(np.uint8)
    regions = np.broadcast_to(regions, (p["N"][2], p["N"][1], p["N"][0])).copy()
    kw = dict(Dind=p["Dind"], Ku1=p["Ku1"], anisU=p["anisU"], B_ext=p["B_ext"], regions=regions)
    free = eng.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], **kw)
    frozen = eng.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], FrozenSpins=[0.0, 1.0], **kw)
    m0 = G.random_unit(p["N"], 3)
    for s in (free, frozen):
        s.set_m(m0)
    tf = free.torque().cpu().numpy()
    tz = frozen.torque().cpu().numpy()
    sel = regions == 1
    assert np.all(tz[:, sel] == 0)
    assert np.array_equal(tz[:, ~sel], tf[:, ~sel])
    frozen.steps(10)
    m = frozen.get_m().cpu().numpy().reshape(m0.shape)
    mn = m0 / np.linalg.norm(m0, axis=0)
    assert np.abs(m[:, sel] - mn[:, sel]).max() < 1e-6
    assert np.abs(m[:, ~sel] - mn[:, ~sel]).max() > 1e-3


@pytest.mark.parametrize("pbc", [(2, 2, 0), (0, 3, 1)])
def test_pbc_torque_matches_oracle(eng, pbc):
    """SetPBC: wrapped stencils (bit-identical without demag) and the periodic
    demag kernel (1e-5 of the largest torque)."""
    p = multilayer_small(N=(16, 12, 4))
    kw = dict(Dind=p["Dind"], Ku1=p["Ku1"], anisU=p["anisU"], B_ext=p["B_ext"])
    m = G.random_unit(p["N"], 8)
    for demag in (False, True):
        g = eng.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], demag=demag, pbc=pbc, **kw)
        o = O.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], demag=demag, pbc=pbc, **kw)
        g.set_m(m)
        o.set_m(m)
        t = g.torque().cpu().numpy()
        to = o.torque()
        if demag:
            assert np.abs(t - to).max() <= 1e-5 * np.abs(to).max()
        else:
            assert np.array_equal(t, to)
        g.free()


@pytest.mark.parametrize("geom", [False, True])
def test_no_demag_spins_matches_oracle(eng, geom):
    """engine/demag.go:67-98 NoDemagSpins: region 1 neither makes nor feels
    demag field (with and without a geometry mask), against the oracle."""
    N, cell = (48, 40, 2), (3e-9, 3e-9, 2e-9)
    regions = np.zeros((2, 40, 48), np.uint8)
    regions[:, :, 30:] = 1
    regions[:, :8, :] = 2
    vol = None
    if geom:
        vol = np.ones((2, 40, 48), np.float32)
        vol[:, 30:, :10] = 0
    kw = dict(Ku1=3e5, anisU=(0, 0, 1), B_ext=(0.01, 0, 0.02), regions=regions, NoDemagSpins=[0, 1, 0],
              FrozenSpins=[0, 0, 1])
    g = eng.Simulation(N, cell, 8e5, 1.3e-11, 0.1, geom=vol, **kw)
    o = O.Simulation(N, cell, 8e5, 1.3e-11, 0.1, vol=vol, **kw)
    m = G.random_unit(N, 3)
    g.set_m(m)
    o.set_m(m)
    t, b = g.torque(beff=True)
    t_o, b_o = o.torque(beff=True)
    b, t = b.cpu().numpy(), t.cpu().numpy()
    assert np.abs(b - b_o).max() <= 1e-5 * np.abs(b_o).max()
    assert np.abs(t - t_o).max() <= 1e-5 * np.abs(t_o).max()
    # region 1 feels no demag field: B_eff there equals the field without demag
    nd = eng.Simulation(N, cell, 8e5, 1.3e-11, 0.1, geom=vol, demag=False, **kw)
    nd.set_m(m)
    _, b_nd = nd.torque(beff=True)
    r1 = np.broadcast_to(regions == 1, b.shape)
    assert np.array_equal(b[r1], b_nd.cpu().numpy()[r1])
    assert np.all(t[np.broadcast_to(regions == 2, t.shape)] == 0)  # FrozenSpins region 2
    g.free()
    nd.free()


def test_launch_shapes_do_not_change_results(eng, tmp_path):
    """Every launch shape the autotuner may choose -- including the torque
    kernel's TMA tiles against its global loads -- gives the same
    trajectory, bit for bit (per-cell arithmetic, max reductions); the
    autotuner's choice is one of its candidates and is cached."""
    from umagnus_b200 import autotune
    p = multilayer_small()
    m = G.random_unit(p["N"], 4)
    shapes = [autotune.DEFAULT,
              {"torque_block": [64, 4], "stage_threads": 128, "stage_waves": 2, "err_waves": 16, "torque_tma": 1},
              {"torque_block": [32, 8], "stage_threads": 256, "stage_waves": 8, "err_waves": 4, "torque_tma": 0},
              {"torque_block": [128, 2], "stage_threads": 64, "stage_waves": 1, "err_waves": 1, "torque_tma": 1},
              {"torque_block": [256, 1], "stage_threads": 64, "stage_waves": 1, "err_waves": 1, "torque_tma": 0}]
    out = []
    for t in shapes:
        g = eng.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], Dind=p["Dind"], Ku1=p["Ku1"],
                           anisU=p["anisU"], B_ext=p["B_ext"])
        g.set_tuning(t)
        assert g.get_tuning() == t
        g.set_m(m)
        g.steps(20)
        out.append((g.get_m().cpu(), g.state()))
        g.free()
    for mm, st in out[1:]:
        assert torch.equal(mm, out[0][0])
        assert st["nsteps"] == out[0][1]["nsteps"] and st["time"] == out[0][1]["time"]
    g = eng.Simulation(p["N"], p["cell"], p["Ms"], p["Aex"], p["alpha"], Dind=p["Dind"], Ku1=p["Ku1"],
                       anisU=p["anisU"], B_ext=p["B_ext"])
    g.set_m(m)
    m_before = g.get_m().clone()
    cache = str(tmp_path / "tuning.json")
    best, log = g.autotune(cache_path=cache)
    assert log is not None and tuple(best["torque_block"]) in autotune.torque_blocks(p["N"][0])
    assert (best["stage_threads"], best["stage_waves"]) in autotune.STAGE_SHAPES
    assert torch.equal(g.get_m(), m_before)  # the search restored m and the time
    assert g.state()["time"] == 0.0
    again, log2 = g.autotune(cache_path=cache)
    assert log2 is None and again == best
    g.steps(20)
    assert torch.equal(g.get_m().cpu(), out[0][0])
    with pytest.raises(Exception):
        g.set_tuning(dict(best, torque_block=[48, 4]))
    g.free()


@pytest.mark.parametrize("openbc", [False, True])
def test_tma_tiles_equal_global_loads_on_awkward_meshes(eng, openbc):
    """The torque kernel's TMA tiles against its global loads, bit for bit,
    on a mesh whose width is not a multiple of the tile (36 cells), with
    holes in the geometry (missing neighbours inside the mesh), interfacial
    DMI with and without OpenBC, anisotropy, Zeeman and 3 layers."""
    from umagnus_b200 import config
    N, cell = (36, 20, 3), (2e-9, 2e-9, 1e-9)
    geom = 1.0 - config.ellipse(N, cell, 14e-9, 10e-9)
    m = G.random_unit(N, 21)
    out = []
    for tma in (1, 0):
        g = eng.Simulation(N, cell, 9e5, 1.3e-11, 0.2, Dind=2e-3, Ku1=4e5, anisU=(0, 0.3, 1), B_ext=(0.01, 0, 0.02),
                           geom=geom, open_bc=openbc)
        t = dict(g.get_tuning(), torque_tma=tma)
        for shape in ([32, 8], [64, 2]):
            g.set_tuning(dict(t, torque_block=shape))
            g.set_m(m)
            tq, b = g.torque(beff=True)
            out.append((tma, shape, tq.cpu(), b.cpu()))
        g.free()
    for tma, shape, tq, b in out[1:]:
        assert torch.equal(tq, out[0][2]) and torch.equal(b, out[0][3]), (tma, shape)
