"""The reference's own regression scripts (test/*.mx3) that use only what
this library implements, run on the GPU engine with the scripts' values and
tolerances (default demag = the brute-force kernel, EnableDemag)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _e():
    from umagnus_b200 import config, engine
    return engine, config


def test_standard_problem_4_relax_and_reversal():
    """test/standardproblem4.mx3: relax to the S state (TOL 1e-5), then 1 ns under
    B_ext = (-24.6, 4.3, 0) mT (TOL 1e-5)."""
    engine, config = _e()
    N = (128, 32, 1)
    cell = (500e-9 / 128, 125e-9 / 32, 3e-9)
    sim = engine.Simulation(N, cell, 800e3, 13e-12, 0.02, B_ext=(0.0, 0.0, 0.0), demag_kernel="brute")
    sim.set_m(config.uniform(N, 1.0, 0.1, 0.0))
    sim.relax()
    np.testing.assert_allclose(sim.average_m(), [0.9669684171676636, 0.1252832127904892, 0.0], rtol=0, atol=1e-5)
    sim.set_B_ext((-24.6e-3, 4.3e-3, 0.0))
    sim.run(1e-9)
    np.testing.assert_allclose(sim.average_m(), [-0.9846124053001404, 0.12604689081287384, 0.04327124357223511],
                               rtol=0, atol=1e-5)
    sim.free()


@pytest.mark.parametrize("dind,want,tol", [(0.0, 0.02785073, 1e-5),          # test/exchange3d.mx3
                                           (1e-20, 0.027852356433868408, 1e-6)])  # test/exchange3d_dmi.mx3
def test_exchange3d_vortex(dind, want, tol):
    engine, config = _e()
    d, n = 100e-9, 32
    N, cell = (n, n, n // 4), (d / n, d / n, d / n)
    sim = engine.Simulation(N, cell, 800e3, 13e-12, 3.0, Dind=dind, demag_kernel="brute")
    sim.set_m(config.vortex(N, cell, 1, 1))
    sim.relax()
    assert abs(sim.average_m()[2] - want) <= tol, sim.average_m()
    sim.free()


def test_dmi_bloch_to_neel():
    """test/dmi.mx3: DMI turns a Bloch wall into a Neel wall (TOL 0.01)."""
    engine, config = _e()
    N = (128, 128, 1)
    cell = (250e-9 / 128, 250e-9 / 128, 0.6e-9)
    sim = engine.Simulation(N, cell, 1100e3, 16e-12, 3.0, Dind=0.1e-3, Ku1=1.27e6, anisU=(0, 0, 1),
                            demag_kernel="brute")
    sim.set_m(config.two_domain(N, cell, (0, 0, -1), (1, 1, 0), (0, 0, 1)))
    sim.relax()
    m = sim.average_m()
    assert abs(m[0] - 0.059) <= 0.01 and abs(m[1] - 0.035) <= 0.01, m
    sim.free()


def _sp4_start(engine, config, solver, demag_kernel="brute", N=(128, 32, 1), cz=3e-9, **kw):
    cell = (500e-9 / 128, 125e-9 / 32, cz)
    sim = engine.Simulation(N, cell, 800e3, 13e-12, 3.0, B_ext=(0.0, 0.0, 0.0), demag_kernel=demag_kernel,
                            solver=solver, **kw)
    sim.set_m(config.uniform(N, 1.0, 0.1, 0.0))
    return sim


def test_rk4_fixed_then_adaptive():
    """test/rk4.mx3: RK4 with alpha 3 for 1 ns, then the reversal field with
    FixDt 1e-14 and alpha 0.02 for 0.1 ns (TOL 1e-3), then FixDt = 0 for 0.4 ns."""
    engine, config = _e()
    sim = _sp4_start(engine, config, engine.RUNGEKUTTA)
    sim.run(1e-9)
    sim.set_solver(FixDt=1e-14)
    sim.set_param("alpha", 0.02)
    sim.set_B_ext((-24.6e-3, 4.3e-3, 0.0))
    sim.run(0.1e-9)
    np.testing.assert_allclose(sim.average_m(), [0.59293, 0.63278, -0.08152], rtol=0, atol=1e-3)
    sim.set_solver(FixDt=0.0)
    sim.run(0.4e-9)
    np.testing.assert_allclose(sim.average_m(), [-0.8740, -0.2713, 0.01795], rtol=0, atol=1e-3)
    sim.free()


def test_euler_after_heun():
    """test/euler.mx3: Heun with alpha 3 for 1 ns, then SetSolver(1) (Euler),
    FixDt 1e-14, alpha 0.02 and the reversal field for 0.1 ns (TOL 1e-3)."""
    engine, config = _e()
    sim = _sp4_start(engine, config, engine.HEUN)
    sim.run(1e-9)
    sim.set_solver(engine.EULER, FixDt=1e-14)
    sim.set_param("alpha", 0.02)
    sim.set_B_ext((-24.6e-3, 4.3e-3, 0.0))
    sim.run(0.1e-9)
    np.testing.assert_allclose(sim.average_m(), [0.59293, 0.63278, -0.08152], rtol=0, atol=1e-3)
    sim.free()


def test_standard_problem_4_newell_3d():
    """test/standardproblem4_newell-3d.mx3: 128x32x2 cells, Newell demag,
    relax then 1 ns reversal with alpha 0.02 (TOL 1e-4)."""
    engine, config = _e()
    sim = _sp4_start(engine, config, engine.DORMANDPRINCE, demag_kernel="newell", N=(128, 32, 2), cz=1.5e-9)
    sim.relax()
    np.testing.assert_allclose(sim.average_m(), [0.9669952392578125, 0.12521563470363617, 0.0], rtol=0, atol=1e-4)
    sim.set_param("alpha", 0.02)
    sim.set_B_ext((-24.6e-3, 4.3e-3, 0.0))
    sim.run(1e-9)
    np.testing.assert_allclose(sim.average_m(), [-0.9841473698616028, 0.13057094812393188, 0.043032702058553696],
                               rtol=0, atol=1e-4)
    sim.free()


def test_frozen_spins_hold_the_state():
    """test/frozenspins.mx3: FrozenSpins = 1 everywhere; neither relax() nor
    the 1 ns reversal moves m from uniform(1, 0.1, 0) (TOL 1e-4)."""
    engine, config = _e()
    sim = _sp4_start(engine, config, engine.DORMANDPRINCE, N=(128, 32, 2), cz=1.5e-9, FrozenSpins=1.0)
    want = [0.9950371980667114, 0.09950374066829681, 0.0]
    sim.relax()
    np.testing.assert_allclose(sim.average_m(), want, rtol=0, atol=1e-4)
    sim.set_param("alpha", 0.02)
    sim.set_B_ext((-24.6e-3, 4.3e-3, 0.0))
    sim.run(1e-9)
    np.testing.assert_allclose(sim.average_m(), want, rtol=0, atol=1e-4)
    sim.free()


def test_dmi_energy_dissipation():
    """test/dmienergy.mx3: 64x64x1 cells of 0.575x0.575x1.15 nm, interfacial
    DMI 3e-3, Ku1 5.9e5 along z, alpha 0.01, m = uniform(1, 1, 1); the total
    energy after 10 ps and 20 ps (expect E1-E0, E2-E0 within 1e-23 J)."""
    engine, config = _e()
    N = (64, 64, 1)
    c, d = 1.15e-9 / 2, 1.15e-9
    sim = engine.Simulation(N, (c, c, d), 6e5, 20e-12, 0.01, Dind=3e-3, Ku1=5.9e5, anisU=(0, 0, 1),
                            demag_kernel="brute")
    sim.set_m(config.uniform(N, 1, 1, 1))
    E0 = sim.energies()["total"]
    sim.run(10e-12)
    E1 = sim.energies()["total"]
    sim.run(10e-12)
    E2 = sim.energies()["total"]
    sim.free()
    assert abs((E1 - E0) - (-2.62692723e-20)) <= 0.001e-20, (E1 - E0)
    assert abs((E2 - E0) - (-4.93337113e-20)) <= 0.001e-20, (E2 - E0)


def test_zeeman_energy():
    """test/zeemanenergy.mx3: E_zeeman = -B.M V for B along +x, +y, -x (tol B Ms V / 1e5)."""
    engine, config = _e()
    N, cell = (128, 32, 2), (5e-9, 4e-9, 3e-9)
    Ms, B = 100e3, 1e-3
    V = N[0] * N[1] * N[2] * cell[0] * cell[1] * cell[2]
    sim = engine.Simulation(N, cell, Ms, 0.0, 0.0, B_ext=(0.0, 0.0, 0.0), demag_kernel="brute")
    sim.set_m(config.uniform(N, 1, 0, 0))
    tol = B * Ms * V / 1e5
    for b, want in (((B, 0, 0), -B * Ms * V), ((0, B, 0), 0.0), ((-B, 0, 0), B * Ms * V)):
        sim.set_B_ext(b)
        assert abs(sim.energies()["zeeman"] - want) <= tol
    sim.free()


def test_relax_from_unstable_equilibrium():
    """test/regression017.mx3: 5x1x1 cells, Ku1 1.3e6 along z; relax() from
    +z and then from -z (the second used to trip the solver: zero error
    must not give a NaN step correction, engine/run.go:156-160)."""
    engine, config = _e()
    N = (5, 1, 1)
    sim = engine.Simulation(N, (1e-9, 1e-9, 1e-9), 1000e3, 10e-12, 0.02, Ku1=1.3e6, anisU=(0, 0, 1),
                            demag_kernel="brute")
    for mz, steps in ((1.0, 87), (-1.0, 174)):
        sim.set_m(config.uniform(N, 0, 0, mz))
        sim.relax()
        assert sim.state()["status"] == 0 and sim.state()["nsteps"] == steps  # as the oracle does
        np.testing.assert_allclose(sim.average_m(), [0, 0, mz], rtol=0, atol=1e-6)
    sim.free()


def _avg_demag(sim, m):
    sim.set_m(m)
    _, b = sim.torque(beff=True)  # no exchange field for uniform m, no other terms: B_eff = B_demag
    return b.double().mean(dim=(1, 2, 3)).cpu().numpy()


@pytest.mark.parametrize("N,cell,pbc,tol_diag,tol_off,want", [
    ((128, 128, 1), (1e-9, 1e-9, 0.5e-9), (0, 0, 0), (1e-2, 1e-2, 2e-2), 1e-9, (0, 0, -1)),       # demag2D.mx3
    ((64, 48, 2), (1e-9, 1.2e-9, 0.5e-9), (0, 0, 0), (3e-2, 3e-2, 6e-2), 1e-9, (0, 0, -1)),       # demag3Dfilm.mx3
    ((128, 2, 1), (1e-9, 1e-9, 0.5e-9), (0, 32, 0), (1e-2, 1e-2, 2e-2), 1e-9, (0, 0, -1)),        # demag2Dpbc.mx3
    ((2, 2, 64), (1e-9, 1e-9, 2e-9), (0, 0, 0), (1e-2, 1e-2, 1e-2), 1e-2, (-0.496, -0.496, 0)),    # demagrod.mx3
    ((2, 2, 2), (1e-9, 1e-9, 2e-9), (0, 0, 16), (1e-2, 1e-2, 1e-2), 1e-2, (-0.496, -0.496, 0)),    # demagrodpbc.mx3
], ids=["demag2D", "demag3Dfilm", "demag2Dpbc", "demagrod", "demagrodpbc"])
def test_demag_tensor_of_films_and_rods(N, cell, pbc, tol_diag, tol_off, want):
    """Average B_demag of uniform m along x, y, z with Msat = 1/mu0 (the
    demag tensor's diagonal) for the reference's film and rod scripts, brute
    force kernel (EnableDemag)."""
    engine, config = _e()
    sim = engine.Simulation(N, cell, 1 / (4e-7 * np.pi), 0.0, 0.0, demag_kernel="brute", pbc=pbc)
    for i in range(3):
        u = [0.0, 0.0, 0.0]
        u[i] = 1.0
        avg = _avg_demag(sim, config.uniform(N, *u))
        for j in range(3):
            if i == j:
                assert abs(avg[j] - want[i]) <= tol_diag[i], (i, avg)
            else:
                assert abs(avg[j]) <= tol_off, (i, j, avg)
    sim.free()


@pytest.mark.parametrize("shifted", [True, False])
def test_pbc_exchange_wrapping(shifted):
    """test/pbc1.mx3: SetPBC(2, 2, 0), 128x64 cells of 5 nm, a 64x32-cell
    rectangle repeated with the mesh period, translated by half a period (the
    magnet split over the four corners) or not; 1 ns with alpha 1 from
    uniform(1, 0.1, 0.01) gives the same <m> either way (TOL 1e-3)."""
    engine, config = _e()
    Nx, Ny, c = 128, 64, 5e-9
    N, cell = (Nx, Ny, 1), (c, c, c)
    shift = (Nx / 2 * c, Ny / 2 * c, 0) if shifted else (0, 0, 0)
    geom = config.rect(N, cell, Nx / 2 * c, Ny / 2 * c, repeat=(Nx * c, Ny * c, 0), transl=shift)
    sim = engine.Simulation(N, cell, 1000e3, 10e-12, 1.0, geom=geom, demag_kernel="brute", pbc=(2, 2, 0))
    sim.set_m(config.uniform(N, 1, 0.1, 0.01))
    sim.run(1e-9)
    np.testing.assert_allclose(sim.average_m(), [0.89947968, 0.23352228, -0.00010287], rtol=0, atol=1e-3)
    sim.free()


def test_gammall_reassigned_late():
    """test/gammaLL.mx3: Heun, MaxErr 1e-4, 16x16x1 cells of 5 nm, B = 1 T
    along z, alpha 0.001; 0.1 ns, then GammaLL doubled, 0.1 ns more
    (TOL 1.2e-4).  The script's table autosave does not touch the time step
    (only Run's stop time is an alarm, engine/run.go:181-192)."""
    engine, config = _e()
    N, c = (16, 16, 1), 5e-9
    sim = engine.Simulation(N, (c, c, c), 1 / (4e-7 * np.pi), 10e-12, 0.001, B_ext=(0, 0, 1.0),
                            demag_kernel="brute", solver=engine.HEUN, MaxErr=1e-4)
    sim.set_m(config.uniform(N, 1, 1, 1))
    sim.run(0.1e-9)
    sim.set_solver(GammaLL=2 * engine.GAMMA_LL)
    sim.run(0.1e-9)
    np.testing.assert_allclose(sim.average_m(), [-0.286423, -0.746625, 0.5970549], rtol=0, atol=1.2e-4)
    sim.free()


def test_no_demag_spins():
    """test/nodemagspins.mx3: 128x32x1 SP4 film, m = uniform(1, 1, 1), region
    0 for x < 0 and 1 for x >= 0; region averages of B_demag with NoDemagSpins
    off, on in region 1, on in both; then with the half y >= 0 cut out of the
    geometry as region 2 (TOL 1e-4; masked regions exactly 0)."""
    engine, config = _e()
    N = (128, 32, 1)
    cell = (500e-9 / 128, 125e-9 / 32, 3e-9)
    X, Y, _ = config.coords(N, cell)
    regions = np.where(X >= 0, 1, 0).astype(np.uint8)
    air = Y >= 0
    regions_air = np.where(air, 2, regions).astype(np.uint8)

    def region_avgs(nodemag, regs, geom=None):
        sim = engine.Simulation(N, cell, 800e3, 0.0, 0.0, regions=regs, geom=geom, demag_kernel="brute",
                                NoDemagSpins=nodemag)
        avg = _avg_by_region(sim, config.uniform(N, 1, 1, 1), regs)
        sim.free()
        return avg

    full = [-0.005299, -0.022127, -0.552248]
    a = region_avgs(None, regions)
    np.testing.assert_allclose(a[0], full, rtol=0, atol=1e-4)
    np.testing.assert_allclose(a[1], full, rtol=0, atol=1e-4)
    a = region_avgs([0, 1], regions)
    np.testing.assert_allclose(a[0], [-0.0103589, -0.02122757, -0.5480939], rtol=0, atol=1e-4)
    assert np.all(a[1] == 0)
    a = region_avgs([1, 1], regions)
    assert np.all(a[0] == 0) and np.all(a[1] == 0)
    geom = (~air).astype(np.float32)
    a = region_avgs([1, 1], regions_air, geom)
    assert all(np.all(a[r] == 0) for r in range(3))
    a = region_avgs([0, 0], regions_air, geom)
    half = [-0.0046074, -0.0391400, -0.53594726]
    np.testing.assert_allclose(a[0], half, rtol=0, atol=1e-4)
    np.testing.assert_allclose(a[1], half, rtol=0, atol=1e-4)
    np.testing.assert_allclose(a[2], [-0.000692, 0.0170129, -0.01630170], rtol=0, atol=1e-4)


def _avg_by_region(sim, m, regions):
    """B_eff (= B_demag: uniform m, no exchange, no other terms) averaged over
    the cells of each region, as Region(r).Average() does (engine/oneregion.go:62-70)."""
    sim.set_m(m)
    _, b = sim.torque(beff=True)
    b = b.double().cpu().numpy().reshape(3, -1)
    reg = np.asarray(regions).ravel()
    return {int(r): b[:, reg == r].mean(axis=1) for r in np.unique(reg)}


@pytest.mark.parametrize("which", ["Ku1", "Ku2"])  # test/anisenergy.mx3, test/anisenergy2.mx3
def test_anisotropy_energy_conservation_without_damping(which):
    """test/anisenergy.mx3 (Ku1 1e6) and anisenergy2.mx3 (Ku2 1e6): 32x10x2
    cells (1, 2, 3 nm), no demag, axis z; the energy change over 1 ns with
    alpha = 0 is below 1e-6 of the change with alpha = 1."""
    engine, config = _e()
    N, c = (32, 10, 2), 1e-9
    sim = engine.Simulation(N, (c, 2 * c, 3 * c), 1000e3, 10e-12, 1.0, anisU=(0, 0, 1), demag=False,
                            **{which: 1e6})
    sim.set_m(config.uniform(N, 1, 0, 0.1))
    E0 = sim.energies()["total"]
    sim.run(1e-9)
    d1 = sim.energies()["total"] - E0
    sim.set_m(config.uniform(N, 1, 0, 0.1))
    E0 = sim.energies()["total"]
    sim.set_param("alpha", 0.0)
    sim.run(1e-9)
    d2 = sim.energies()["total"] - E0
    sim.free()
    assert abs(d2 / d1) <= 1e-6, (d1, d2)


@pytest.mark.parametrize("extra", [{}, {"Ku2": 2e5}, {"Kc2": 1e3}, {"Kc3": 1e3}],
                         ids=["anisenergyconservation", "2_Ku2", "3_Kc2", "4_Kc3"])
def test_cubic_and_uniaxial_energy_conservation(extra):
    """test/anisenergyconservation.mx3 and its variants 2-4 (adding Ku2 2e5,
    Kc2 1e3 or Kc3 1e3): one cell, Kc1 1e3 and Ku1 1e5 along (1, 1, 0), alpha
    1e-6, MaxDt 1e-13; the total energy stays within 1e-5 (relative) over
    ten runs of 10 ps."""
    engine, config = _e()
    N = (1, 1, 1)
    sim = engine.Simulation(N, (1e-9, 1e-9, 1e-9), 1000e3, 0.0, 1e-6, Ku1=1e5, anisU=(1, 1, 0), Kc1=1e3,
                            anisC1=(1, 0, 0), anisC2=(0, 1, 0), demag=False, MaxDt=1e-13, **extra)
    sim.set_m(config.uniform(N, 0.3, 0.7, 0.1))
    E0 = sim.energies()["total"]
    for _ in range(10):
        sim.run(10e-12)
        E = sim.energies()["total"]
        assert abs((E0 - E) / E0) <= 1e-5, (E0, E)
    sim.free()


def test_cubic_anisotropy_against_field():
    """test/cubicanisotropy.mx3: 64x64x1 disc, Kc1 0.2e6 with AnisC1 =
    (100, 0, 0) (unnormalised), relaxed under B along (1, 1, 0); the OOMMF
    values of <m> within 1e-3."""
    engine, config = _e()
    N, cell = (64, 64, 1), (4e-9, 4e-9, 2e-9)
    geom = config.ellipse(N, cell, 64 * 4e-9, 64 * 4e-9)
    sim = engine.Simulation(N, cell, 1100e3, 13e-12, 1.0, B_ext=(0.0, 0.0, 0.0), geom=geom, Kc1=0.2e6,
                            anisC1=(100, 0, 0), anisC2=(0, 1, 0), demag_kernel="brute")
    sim.set_m(config.uniform(N, 1, 0, 0))
    for b, want in ((0.0, (1, 0, 0)), (0.01, (0.9994, 0.0270, 0)), (0.03, (0.9967, 0.0776, 0)),
                    (0.10, (0.9711, 0.2367, 0)), (0.30, (0.7040, 0.7040, 0))):
        sim.set_B_ext((b, b, 0.0))
        sim.relax()
        np.testing.assert_allclose(sim.average_m(), want, rtol=0, atol=1e-3, err_msg=f"B={b}")
    sim.free()


def test_uniaxial_anisotropy_against_field():
    """test/uniaxialanisotropy.mx3: 64x64x1 film, Ku1 = +-0.5e6 along x,
    relaxed under B; the OOMMF values within 1e-3, AnisU = (100, 0, 0) the
    same as (1, 0, 0), and Ku1 = -1e6 along z keeps m in the plane."""
    engine, config = _e()
    N, cell = (64, 64, 1), (4e-9, 4e-9, 2e-9)
    sim = engine.Simulation(N, cell, 1100e3, 13e-12, 1.0, B_ext=(0.0, 0.0, 0.0), Ku1=0.5e6, anisU=(1, 0, 0),
                            demag_kernel="brute")
    sim.set_m(config.uniform(N, 1, 1, 0))

    def relaxed(B, comp, want):
        sim.set_B_ext(B)
        sim.relax()
        assert abs(sim.average_m()[comp] - want) <= 1e-3, (B, sim.average_m())

    for by, want in ((0.0, 0.0), (0.01, 0.011), (0.03, 0.033), (0.10, 0.110), (0.30, 0.331)):
        relaxed((0, by, 0), 1, want)
    sim.set_param("Ku1", -0.5e6)
    relaxed((0, 0, 0), 1, 1.0)
    relaxed((0.01, 0, 0), 0, 0.011)
    relaxed((0.10, 0, 0), 0, 0.110)
    sim.set_param("anisU", (100, 0, 0))
    relaxed((0.10, 0, 0), 0, 0.110)
    sim.set_param("anisU", (0, 0, 1))
    sim.set_param("Ku1", -1e6)
    relaxed((0, 0, 0), 2, 0.0)
    sim.free()


def test_standard_problem_4b():
    """test/standardproblem4b.mx3: relax with alpha 0.02, then 1 ns under
    B_ext = (-35.5, -6.3, 0) mT (TOL 1e-3)."""
    engine, config = _e()
    N = (128, 32, 1)
    cell = (500e-9 / 128, 125e-9 / 32, 3e-9)
    sim = engine.Simulation(N, cell, 800e3, 13e-12, 0.02, B_ext=(0.0, 0.0, 0.0), demag_kernel="brute")
    sim.set_m(config.uniform(N, 1.0, 0.1, 0.0))
    sim.relax()
    np.testing.assert_allclose(sim.average_m(), [0.9669684171676636, 0.1252732276916504, 0], rtol=0, atol=1e-3)
    sim.set_B_ext((-35.5e-3, -6.3e-3, 0.0))
    sim.run(1e-9)
    np.testing.assert_allclose(sim.average_m(), [-0.9692331552505493, -0.11889542198181152, -0.0053076110780239105],
                               rtol=0, atol=1e-3)
    sim.free()


def test_bulk_dmi_rotation_symmetry():
    """test/dmibulksymm.mx3: 16^3 cube with bulk DMI 1e-3; 0.1 ns from m along
    x, y, z (and from (0,1,1), (1,0,1), (1,1,0)) gives the rotated averages
    (TOL 1e-4)."""
    engine, config = _e()
    N, c = (16, 16, 16), 2e-9
    sim = engine.Simulation(N, (c, c, c), 1e6, 10e-12, 1.0, Dbulk=1e-3, demag_kernel="brute")

    def run_from(*m):
        sim.set_m(config.uniform(N, *m))
        sim.run(1e-10)
        return sim.average_m()

    m0 = run_from(1, 0, 0)
    assert abs(run_from(0, 1, 0)[1] - m0[0]) <= 1e-4
    assert abs(run_from(0, 0, 1)[2] - m0[0]) <= 1e-4
    m0 = run_from(0, 1, 1)
    assert abs(run_from(1, 0, 1)[1] - m0[0]) <= 1e-4
    assert abs(run_from(1, 1, 0)[2] - m0[0]) <= 1e-4
    sim.free()


def test_energy_density_integrates_to_energy():
    """test/edens.mx3 (total): 200x50x2 ellipse in two regions with their own
    Aex, Msat and Ku1, AnisU (1, 2, 3), Kc1 2e5, B_ext 1 mT along z, vortex,
    0.1 ns with alpha 1; mesh volume x average of Edens_total = E_total
    within 1e-3."""
    engine, config = _e()
    N, cell = (200, 50, 2), (5e-9, 4e-9, 3e-9)
    X, _, _ = config.coords(N, cell)
    regions = np.where(X < 0, 1, 2).astype(np.uint8)
    aex = np.zeros(256)
    aex[1], aex[2] = 10e-12, 13e-12
    Ms = np.where(regions == 1, 1e6, 0.8e6).astype(np.float32)
    Ku1 = np.where(regions == 1, 1e5, -2e5).astype(np.float32)
    sim = engine.Simulation(N, cell, Ms, aex, 1.0, Ku1=Ku1, anisU=(1, 2, 3), Kc1=2e5, anisC1=(1, 0, 0),
                            anisC2=(0, 1, 0), B_ext=(0, 0, 1e-3), regions=regions,
                            geom=config.ellipse(N, cell, 1e-6, 200e-9), demag_kernel="brute")
    sim.set_m(config.vortex(N, cell, 1, 1))
    sim.run(0.1e-9)
    volume = 1e-6 * 200e-9 * 6e-9
    avg = sim.energy_density().double().mean().item()
    E = sim.energies()["total"]
    sim.free()
    assert abs(volume * avg / E - 1) <= 1e-3, (volume * avg, E)



def test_dmi_bloch_to_neel_along_y():
    """test/dmiY.mx3: test/dmi.mx3 rotated by 90 degrees (TwoDomain(...).RotZ(pi/2)),
    MaxDt 5e-13, 5 ns: <m> = (-0.035, 0.059) within 0.01."""
    engine, config = _e()
    N = (128, 128, 1)
    cell = (250e-9 / 128, 250e-9 / 128, 0.6e-9)
    sim = engine.Simulation(N, cell, 1100e3, 16e-12, 3.0, Dind=0.1e-3, Ku1=1.27e6, anisU=(0, 0, 1), MaxDt=5e-13,
                            demag_kernel="brute")
    sim.set_m(config.sample(N, cell, config.rot_z(config.two_domain_fn(cell, (0, 0, -1), (1, 1, 0), (0, 0, 1)),
                                                  np.pi / 2)))
    sim.run(5e-9)
    m = sim.average_m()
    sim.free()
    assert abs(m[0] + 0.035) <= 0.01 and abs(m[1] - 0.059) <= 0.01, m


def test_dmi_3d_wall_cell():
    """test/dmi3d.mx3: 64x64x2 cells (0.6, 0.6, 0.3 nm), DMI + exchange +
    Ku1, two-domain start, 0.5 ns: m in cell (32, 32, 0) = (0.8979, 0.3989,
    0.1859) within 1e-3 (the reference's 2D solution)."""
    engine, config = _e()
    N, c = (64, 64, 2), 0.6e-9
    cell = (c, c, c / 2)
    sim = engine.Simulation(N, cell, 1100e3, 16e-12, 3.0, Dind=0.1e-3, Ku1=1.27e6, anisU=(0, 0, 1),
                            demag_kernel="brute")
    sim.set_m(config.two_domain(N, cell, (0, 0, -1), (1, 1, 0), (0, 0, 1)))
    sim.run(0.5e-9)
    m = sim.get_m().cpu().numpy()[:, 0, 32, 32]
    sim.free()
    np.testing.assert_allclose(m, [0.8979, 0.3989, 0.1859], rtol=0, atol=1e-3)


def test_cubic_anisotropy_energy_of_one_cell():
    """test/cubic_full.mx3: E_anis / V of one cell at theta 23, phi 11 degrees
    for Kc1, Kc2, Kc3 = +-1e6 alone (TOL 1e-2 J/m^3)."""
    engine, config = _e()
    N, V = (1, 1, 1), 1e-27
    th, ph = np.deg2rad(23), np.deg2rad(11)
    sim = engine.Simulation(N, (1e-9, 1e-9, 1e-9), 1000e3, 0.0, 0.0, Kc1=1e6, anisC1=(1, 0, 0), anisC2=(0, 1, 0),
                            demag=False)
    sim.set_m(config.uniform(N, np.sin(ph) * np.cos(th), np.sin(ph) * np.sin(th), np.cos(ph)))
    for k, want in (("Kc1", 35254.007), ("Kc2", 165.23309326171875), ("Kc3", 912.3794555664062)):
        for sign in (1, -1):
            for kk in ("Kc1", "Kc2", "Kc3"):
                sim.set_param(kk, sign * 1e6 if kk == k else 0.0)
            e = sim.energies()["anisotropy"] / V
            assert abs(e - sign * want) <= 1e-2, (k, sign, e)
    sim.free()


def test_uniaxial_anisotropy_energy_of_one_cell():
    """test/uniaxial_full.mx3: E_anis / V of one cell at 17 degrees from the
    x easy axis for Ku2 = +-1e6 and Ku1 = +-1e6 alone (TOL 1 J/m^3)."""
    engine, config = _e()
    N, V = (1, 1, 1), 1e-27
    th = np.deg2rad(17)
    sim = engine.Simulation(N, (1e-9, 1e-9, 1e-9), 1000e3, 0.0, 0.0, Ku2=1e6, anisU=(1, 0, 0), demag=False)
    sim.set_m(config.uniform(N, np.cos(th), np.sin(th), 0))
    for ku1, ku2, want in ((0, 1e6, -836344.9375), (0, -1e6, 836344.9375), (1e6, 0, -914519), (-1e6, 0, 914519)):
        sim.set_param("Ku1", ku1)
        sim.set_param("Ku2", ku2)
        e = sim.energies()["anisotropy"] / V
        assert abs(e - want) <= 1, (ku1, ku2, e)
    sim.free()


@pytest.mark.parametrize("ms", [(3.2, 4.6, 3.9, 7.8), (1.1, 1.1, 1.1, 1.1)])
def test_exchange_inhomo_against_oommf(ms):
    """test/exchange_inhomo.mx3: per-region Aex (harmonic mean between
    regions) and Msat on the random 4x4x1 state of testdata/randommag4x4x1.ovf
    (tests/golden); E_exch = OOMMF's 154.4891365 J within 1e-5, independent of
    Msat."""
    from tests.test_oracle_energy import _exchange_inhomo_case
    engine, config = _e()
    N, cell, m, regions, aex = _exchange_inhomo_case()
    Ms = np.asarray((0.0,) + tuple(ms), np.float32)[regions]
    sim = engine.Simulation(N, cell, Ms, aex, 0.1, regions=regions, demag=False)
    sim.set_m(m)
    E = sim.energies()["exchange"]
    sim.free()
    assert abs(E - 154.4891365) <= 1e-5, E


def test_antiferromagnetic_interexchange():
    """test/interexchange.mx3: the SP4 film split at y = 0 into regions 1
    (y >= 0) and 2 (y < 0), ext_ScaleExchange(1, 2, -1) (antiferromagnetic
    coupling), alpha 3, 10 ns: <m> = (0, 0.114170685410499, 0) within 1e-5."""
    engine, config = _e()
    N = (128, 32, 1)
    cell = (500e-9 / 128, 125e-9 / 32, 3e-9)
    _, Y, _ = config.coords(N, cell)
    regions = np.where(Y >= 0, 1, 2).astype(np.uint8)
    sim = engine.Simulation(N, cell, 800e3, 13e-12, 3.0, regions=regions, exchange_scale={(1, 2): -1.0},
                            demag_kernel="brute")
    sim.set_m(config.uniform(N, 1, 0.1, 0))
    sim.run(10e-9)
    m = sim.average_m()
    sim.free()
    np.testing.assert_allclose(m, [0, 0.114170685410499, 0], rtol=0, atol=1e-5)


def test_demag_with_regions():
    """test/demagRegion.mx3: 64x64x2 film (1, 1, 0.5 nm) in three regions
    (x >= 0, x < 0, an ellipse) all with Msat = 2/mu0: the averaged B_demag of
    uniform m along x, y, z is (0 +- 0.1, off-diagonal 1e-8, -2 +- 0.1); with
    Msat = 1/mu0, B_demag_z of m along z is -1 +- 0.1."""
    engine, config = _e()
    N, cell = (64, 64, 2), (1e-9, 1e-9, 0.5e-9)
    X, _, _ = config.coords(N, cell)
    regions = np.where(X >= 0, 1, 2).astype(np.uint8)
    regions[config.ellipse(N, cell, 10e-9, 20e-9) > 0] = 3
    mu0 = 4e-7 * np.pi
    Ms = np.full(regions.shape, 2 / mu0, np.float32)
    sim = engine.Simulation(N, cell, Ms, 0.0, 0.0, regions=regions, demag_kernel="brute")
    for i, want in ((0, 0.0), (1, 0.0), (2, -2.0)):
        u = [0.0, 0.0, 0.0]
        u[i] = 1.0
        avg = _avg_demag(sim, config.uniform(N, *u))
        assert abs(avg[i] - want) <= 0.1, (i, avg)
        assert all(abs(avg[j]) <= 1e-8 for j in range(3) if j != i), (i, avg)
    sim.set_param("Msat", 1 / mu0)
    assert abs(_avg_demag(sim, config.uniform(N, 0, 0, 1))[2] + 1.0) <= 0.1
    sim.free()


def test_standard_problem_4_brute_3d():
    """test/standardproblem4-3d.mx3: 128x32x2 cells, brute-force demag
    (EnableDemag), relax then the 1 ns reversal with alpha 0.02 (TOL 1e-4)."""
    engine, config = _e()
    sim = _sp4_start(engine, config, engine.DORMANDPRINCE, N=(128, 32, 2), cz=1.5e-9)
    sim.relax()
    np.testing.assert_allclose(sim.average_m(), [0.9669952392578125, 0.12521563470363617, 0], rtol=0, atol=1e-4)
    sim.set_param("alpha", 0.02)
    sim.set_B_ext((-24.6e-3, 4.3e-3, 0.0))
    sim.run(1e-9)
    np.testing.assert_allclose(sim.average_m(), [-0.9846296310424805, 0.1256464719772339, 0.04335508495569229],
                               rtol=0, atol=1e-4)
    sim.free()


def test_stepper_cache_is_flushed_by_a_new_m():
    """test/steppercache.mx3: one cell, RK45DP with FixDt 1e-12 in 50 mT
    along z; a step from m = +x and a step from m = -x rotate m by the same
    angle (the FSAL torque of the old m must not be reused), TOL 1e-5."""
    engine, config = _e()
    N = (1, 1, 1)
    sim = engine.Simulation(N, (1.0, 1.0, 1.0), 1000e3, 0.0, 0.1, B_ext=(0, 0, 0.05), demag=False,
                            solver=engine.DORMANDPRINCE, FixDt=1e-12)
    sim.set_m(config.uniform(N, 1, 0, 0))
    sim.steps(1)
    want = np.arccos(np.dot([1, 0, 0], sim.average_m()))
    sim.set_m(config.uniform(N, -1, 0, 0))
    sim.steps(1)
    got = np.arccos(np.dot([-1, 0, 0], sim.average_m()))
    sim.free()
    assert abs(got - want) <= 1e-5 and want > 1e-3, (got, want)


def test_run_while():
    """test/runwhile.mx3: a 20x20 disc of 4 nm cells, alpha 1: RunWhile(MaxTorque
    > 1e-3), then B_ext = (0, 0.01, 1) T and RunWhile(<m_y> < 0.5): <m_y> =
    0.53 within 0.02 (the overshoot of the last step).  The condition is
    checked before every step, as engine/run.go:200-231 runWhile does."""
    engine, config = _e()
    N, c = (20, 20, 1), 4e-9
    cell = (c, c, c)
    sim = engine.Simulation(N, cell, 800e3, 13e-12, 1.0, B_ext=(0, 0, 0), geom=config.ellipse(N, cell, 20 * c, 20 * c),
                            demag_kernel="brute")
    sim.set_m(config.uniform(N, 1, 0, 0))

    def max_torque():  # MaxTorque: max |torque| of the current m
        return float(torch.linalg.vector_norm(sim.torque(), dim=0).max())

    n = 0
    while max_torque() > 1e-3 and n < 200000:
        sim.steps(1)
        n += 1
    sim.set_B_ext((0, 0.01, 1.0))
    while sim.average_m()[1] < 0.5 and n < 400000:
        sim.steps(1)
        n += 1
    my = sim.average_m()[1]
    sim.free()
    assert abs(my - 0.53) <= 0.02, (my, n)
