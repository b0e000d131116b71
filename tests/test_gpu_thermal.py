"""Thermal field on the GPU (engine/temperature.go, temperature2.cl):

- the noise generator against its restatement (oracle.thermal_normals, pinned
  to the Philox known answers) and SetTemperature bit for bit against the
  oracle (itself bit-identical to the reference kernel);
- the engine's B_eff with Temp = the field without it + noise x scale;
- the reference's own regression script test/rk4temperature.mx3: 768x768
  independent macrospins (Aex 0, no demag), Ku1 2500 J/m^3 along z, 100 K,
  RK4 with FixDt 2e-12 s for 5 ns: <m> = (0, 0, 0.8366) within 1e-3.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests import golden_pins as G

pytestmark = pytest.mark.gpu
KB = 1.380650424e-23
GAMMA = 1.7595e11


def test_noise_matches_restatement():
    from umagnus_b200 import opencl as cl
    n = 100003
    seed, step = 0xDEADBEEF12345678, 42
    noise = torch.empty((3, n), dtype=torch.float32, device="cuda")
    cl.ThermalNoise(noise, seed, step)
    want = O.thermal_normals(seed, step, n)
    got = noise.cpu().numpy()
    assert np.abs(got - want).max() <= 4e-6 * max(1.0, float(np.abs(want).max()))
    # identical on a second call (counter-based: no state)
    again = torch.empty_like(noise)
    cl.ThermalNoise(again, seed, step)
    assert torch.equal(noise, again)


def test_noise_statistics():
    from umagnus_b200 import opencl as cl
    n = 2_000_000
    noise = torch.empty((3, n), dtype=torch.float32, device="cuda")
    cl.ThermalNoise(noise, 99, 0)
    z = noise.double()
    assert float(z.mean(dim=1).abs().max()) < 5 / np.sqrt(n)
    assert float((z.var(dim=1) - 1).abs().max()) < 8 * np.sqrt(2 / n)
    c = torch.corrcoef(z)
    assert float((c - torch.eye(3, dtype=c.dtype, device=c.device)).abs().max()) < 5 / np.sqrt(n)


def test_set_temperature_bitexact():
    from umagnus_b200 import opencl as cl
    rng = np.random.default_rng(8)
    n = 3001
    noise = rng.standard_normal(n).astype(np.float32)
    Ms = (rng.random(n) * 1e6 + 1e5).astype(np.float32)
    Ms[::17] = 0
    temp = (rng.random(n) * 400).astype(np.float32)
    k2 = float(np.float32(2 * KB / (GAMMA * 1e-24 * 2e-13)))
    want = np.zeros(n, np.float32)
    O.set_temperature(want, noise, k2, Ms, temp, 0.05)
    B = torch.zeros(n, dtype=torch.float32, device="cuda")
    cu = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    cl.SetTemperature(B, cu(noise), k2, cl.MSlice(cu(Ms)), cl.MSlice(cu(temp)), 0.05)
    assert np.array_equal(B.cpu().numpy(), want)


def test_engine_thermal_field():
    """B_eff(T) - B_eff(0) is the noise of step 0 times sqrt(k2 alpha T / Ms),
    k2 = float32(2 kB / ((GammaLL V) dt)) (engine/temperature.go:111)."""
    from umagnus_b200 import engine
    N, cell = (24, 16, 2), (3e-9, 3e-9, 2e-9)
    kw = dict(Ku1=2e5, anisU=(0, 0, 1), B_ext=(0, 0, 0.01), solver=engine.RUNGEKUTTA, FixDt=1e-13)
    hot = engine.Simulation(N, cell, 8e5, 1.3e-11, 0.05, Temp=300.0, ThermSeed=11, **kw)
    cold = engine.Simulation(N, cell, 8e5, 1.3e-11, 0.05, **kw)
    m = G.random_unit(N, 2)
    hot.set_m(m)
    cold.set_m(m)
    _, bh = hot.torque(beff=True)
    _, bc = cold.torque(beff=True)
    n = N[0] * N[1] * N[2]
    k2 = np.float32(2 * KB / (GAMMA * (cell[0] * cell[1] * cell[2]) * 1e-13))
    sc = np.sqrt(np.float32(np.float32(np.float32(k2 * np.float32(0.05)) * np.float32(300.0)) * np.float32(1 / 8e5)))
    want = O.thermal_normals(11, 0, n).reshape((3,) + hot.shape) * sc
    diff = (bh - bc).cpu().numpy()
    assert np.abs(diff - want).max() <= 1e-5 * np.abs(want).max()
    # energies carry the thermal term in the total only; relax() runs without noise
    E = hot.energies()
    Et = E["total"] - (((E["anisotropy"] + E["demag"]) + E["exchange"]) + E["zeeman"])
    mm = hot.get_m().cpu().numpy().reshape(want.shape).astype(np.float64)
    Et_want = -(cell[0] * cell[1] * cell[2]) * 8e5 * float(np.sum(mm * want))  # engine/temperature.go:124-130
    assert abs(Et - Et_want) <= 1e-3 * abs(Et_want) + 1e-6 * abs(E["total"])
    hot.relax()
    cold.relax()
    assert np.allclose(hot.average_m(), cold.average_m(), atol=1e-6)
    hot.free()
    cold.free()


def test_rk4temperature_regression():
    """test/rk4temperature.mx3."""
    from umagnus_b200 import config, engine
    N, c = (768, 768, 1), 10e-9
    sim = engine.Simulation(N, (c, c, c), 1e6, 0.0, 0.1, Ku1=1e4 / 4, anisU=(0, 0, 1), demag=False,
                            solver=engine.RUNGEKUTTA, FixDt=2e-12, Temp=100.0, ThermSeed=20240101)
    sim.set_m(config.uniform(N, 0, 0, 1))
    sim.run(5e-9)
    avg = sim.average_m()
    assert abs(avg[0]) < 1e-3 and abs(avg[1]) < 1e-3
    assert abs(avg[2] - 0.8366) < 1e-3, avg
    sim.free()
