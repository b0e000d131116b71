"""The reference's own regression scripts (test/*.mx3) that use only what
this library implements, run on the GPU engine with the scripts' values and
tolerances (default demag = the brute-force kernel, EnableDemag)."""
import numpy as np
import pytest

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
