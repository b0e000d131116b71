"""Energies and Relax() on the GPU engine (through the C-ABI), against the
oracle and against the reference's own regression pins:

- test/standardproblem4b_newell.mx3: relax() to the S state, then a 1 ns
  reversal under B_ext = (-35.5, -6.3, 0) mT (RK45DP), <m> within 1e-3;
- test/energy.mx3: energy differences between a relaxed vortex and the state
  relaxed under 100 mT, against the OOMMF figures quoted there.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_pins as G

pytestmark = pytest.mark.gpu


def _engine():
    from umagnus_b200 import config, engine
    return engine, config


def test_energies_match_oracle():
    """Each energy term of a random state (DMI, K1 + K2, Zeeman, demag, an
    elliptical geometry) within 1e-5 of the FP64 oracle."""
    engine, config = _engine()
    N, cell = (24, 20, 4), (2e-9, 2.5e-9, 1.5e-9)
    geom = config.ellipse(N, cell, N[0] * cell[0], N[1] * cell[1])
    kw = dict(Dind=2e-3, Ku1=3e5, Ku2=1e5, anisU=(0.2, 0.3, 0.9), B_ext=(0.01, -0.02, 0.05))
    sim = engine.Simulation(N, cell, 9e5, 1.2e-11, 0.1, geom=geom, **kw)
    sim.set_m(G.random_unit(N, 21))
    m = sim.get_m().cpu().numpy()
    E = sim.energies()
    orc = O.Simulation(N, cell, 9e5, 1.2e-11, 0.1, vol=geom, **kw)
    want = O.energies(orc, m)
    scale = sum(abs(want[k]) for k in ("demag", "exchange", "anisotropy", "zeeman"))
    for k in ("demag", "exchange", "anisotropy", "zeeman"):
        assert abs(E[k] - want[k]) <= 1e-5 * abs(want[k]) + 1e-9 * scale, (k, E[k], want[k])
    assert abs(E["total"] - want["total"]) <= 1e-5 * scale
    sim.free()


def test_energy_density_matches_fp64():
    """Edens_total per cell (engine/energy.go:36 SetTotalEdens) of a
    multi-region state with per-cell Ms and easy axes, against the FP64
    instantiation of the oracle (itself pinned to the CPU oracle), and its
    sum against the engine's total energy."""
    import torch
    from oracle import gpu64
    engine, config = _engine()
    N, cell = (32, 24, 4), (2e-9, 2e-9, 2e-9)
    rng = np.random.default_rng(5)
    regions = rng.integers(0, 3, size=(N[2], N[1], N[0])).astype(np.uint8)
    Ms = np.array([6e5, 9e5, 7e5], np.float32)[regions]
    aex = np.zeros(256)
    aex[:3] = [1.0e-11, 1.5e-11, 1.2e-11]
    u = rng.normal(size=(3,) + regions.shape).astype(np.float32)
    sim = engine.Simulation(N, cell, Ms, aex, 0.05, Ku1=2e5, anisU=u, regions=regions, B_ext=(0.0, 0.01, 0.02))
    sim.set_m(G.random_unit(N, 4))
    dens = sim.energy_density().double()
    m = sim.get_m().double()
    ref = gpu64.System64(N, cell, Ms.astype(np.float64), O.exch_lut(aex, dtype=np.float64), regions, 0.05,
                         kernel=O.newell_kernel(N, cell), Ku1=2e5, anisU=u.astype(np.float64),
                         B_ext=(0.0, 0.01, 0.02)).energy_density(m)
    err = float((dens - ref).abs().max() / ref.abs().max())
    assert err < 1e-5, err
    V = cell[0] * cell[1] * cell[2]
    assert float(dens.sum()) * V == pytest.approx(sim.energies()["total"], rel=1e-5)
    sim.free()


def test_relax_matches_oracle():
    """Relax() of a small film from a tilted state: same final <m> (1e-3) and
    energy (1e-4) as the oracle's restatement; time unchanged."""
    engine, config = _engine()
    N, cell = (32, 16, 1), (4e-9, 4e-9, 3e-9)
    kw = dict(Ku1=1e4, anisU=(1.0, 0.0, 0.0))
    m0 = config.uniform(N, 1.0, 1.0, 0.2)
    sim = engine.Simulation(N, cell, 8e5, 1.3e-11, 0.02, **kw)
    sim.set_m(m0)
    t0 = sim.state()["time"]
    sim.relax()
    assert sim.state()["time"] == t0
    orc = O.Simulation(N, cell, 8e5, 1.3e-11, 0.02, **kw)
    orc.set_m(m0)
    O.relax(orc)
    got = np.array(sim.average_m())
    want = orc.m.reshape(3, -1).mean(axis=1)
    assert np.max(np.abs(got - want)) < 1e-3, (got, want)
    e_got, e_want = sim.energies()["total"], O.energies(orc)["total"]
    assert abs(e_got - e_want) <= 1e-4 * abs(e_want)
    sim.free()


def test_standard_problem_4b_newell():
    """test/standardproblem4b_newell.mx3:6-27 (Newell demag)."""
    engine, config = _engine()
    N = (128, 32, 1)
    cell = (500e-9 / 128, 125e-9 / 32, 3e-9)
    sim = engine.Simulation(N, cell, 800e3, 13e-12, 0.02, B_ext=(0.0, 0.0, 0.0))
    sim.set_m(config.uniform(N, 1.0, 0.1, 0.0))
    sim.relax()
    np.testing.assert_allclose(sim.average_m(), [0.9669625163078308, 0.12528464198112488, 0.0], rtol=0, atol=1e-3)
    sim.set_B_ext((-35.5e-3, -6.3e-3, 0.0))
    sim.run(1e-9)
    assert sim.state()["time"] == pytest.approx(1e-9, rel=1e-12)
    np.testing.assert_allclose(sim.average_m(), [-0.9702987670898438, -0.12229042601585388, -0.004722175188362598],
                               rtol=0, atol=1e-3)
    sim.free()


def test_energy_differences_vs_oommf():
    """test/energy.mx3: relax a vortex in a 512x256x40 nm ellipse, relax again
    under B_ext = 100 mT along x; the energy differences match OOMMF's within
    the script's tolerances (1e-18 J, anisotropy 1e-21 J)."""
    engine, config = _engine()
    l, w, d, c = 512e-9, 256e-9, 40e-9, 4e-9
    N, cell = (128, 64, 1), (c, c, d)
    vol = l * w * d * (np.pi / 4)
    geom = config.ellipse(N, cell, l, w)
    sim = engine.Simulation(N, cell, 860e3, 13e-12, 3.0, Ku1=50.0, anisU=(1.0, 0.0, 0.0), geom=geom,
                            B_ext=(0.0, 0.0, 0.0))
    sim.set_m(config.vortex(N, cell, 1, 1))
    sim.relax()
    E1 = sim.energies()
    sim.set_B_ext((100e-3, 0.0, 0.0))
    sim.relax()
    E2 = sim.energies()
    oommf = {"total": (12274.249330 - (-56507.645615)) * vol, "exchange": (5038.693945 - 71.438905) * vol,
             "anisotropy": (19.517039 - 0.271210) * vol, "demag": (7216.038345 - 29186.031229) * vol,
             "zeeman": (0 - (-85765.386961)) * vol}
    tol = {"total": 1e-18, "exchange": 1e-18, "anisotropy": 1e-21, "demag": 1e-18, "zeeman": 1e-18}
    for k in oommf:
        assert abs((E1[k] - E2[k]) - oommf[k]) <= tol[k], (k, E1[k] - E2[k], oommf[k])
    sim.free()
