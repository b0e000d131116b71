"""The FP64 torch instantiation of the oracle (oracle/gpu64.py, the
reference for the precision report at full size) against the CPU oracle's
FP64 variant: torque, effective field, energy density and RK45DP steps on a
small multi-region mesh with per-cell Ms, Ku1 and easy axes.  Runs with
torch on the CPU here; the same code runs on the GPU in the report."""
import numpy as np
import pytest
import torch

from oracle import gpu64
from oracle import oracle as O

N = (12, 10, 3)
CELL = (2e-9, 2e-9, 2e-9)


def case(seed=3):
    rng = np.random.default_rng(seed)
    shape = (N[2], N[1], N[0])
    regions = rng.integers(0, 4, size=shape).astype(np.uint8)
    ms_r = np.array([6e5, 9e5, 6e5, 9e5])
    aex_r = np.zeros(256)
    aex_r[:4] = [1.0e-11, 1.5e-11, 1.0e-11, 1.5e-11]
    u_r = rng.normal(size=(4, 3))
    Ms = ms_r[regions]
    Ku1 = np.full(shape, 2e5)
    u = np.stack([u_r[regions][..., c] for c in range(3)])
    m0 = rng.normal(size=(3,) + shape)
    return regions, Ms, aex_r, Ku1, u, m0


def systems(B_ext=(0.0, 0.01, 0.02)):
    regions, Ms, aex_r, Ku1, u, m0 = case()
    cpu = O.Simulation(N, CELL, Ms, 0.0, 0.05, dtype=np.float64, Ku1=Ku1, anisU=u, B_ext=B_ext, regions=regions,
                       Aex_regions=aex_r)
    K = O.newell_kernel(N, CELL)
    g = gpu64.System64(N, CELL, Ms, O.exch_lut(aex_r, dtype=np.float64), regions, 0.05, kernel=K, Ku1=Ku1,
                       anisU=u, B_ext=B_ext, device="cpu")
    return cpu, g, m0


def test_torque_and_field():
    cpu, g, m0 = systems()
    cpu.set_m(m0)
    tau, B = cpu.torque(beff=True)
    m = torch.as_tensor(cpu.m)
    B64 = g.beff(m).numpy()
    t64 = g.torque(m).numpy()
    assert np.abs(B64 - B).max() <= 1e-12 * np.abs(B).max()
    assert np.abs(t64 - tau).max() <= 1e-12 * np.abs(tau).max()


def test_energy_density_sums_to_the_oracle_energy():
    cpu, g, m0 = systems()
    cpu.set_m(m0)
    E = O.energies(cpu)
    e64 = g.energy_density(torch.as_tensor(cpu.m)).numpy()
    V = CELL[0] * CELL[1] * CELL[2]
    assert e64.sum() * V == pytest.approx(E["total"], rel=1e-12)


def test_rk45dp_steps():
    cpu, g, m0 = systems()
    cpu.set_m(m0)
    st = gpu64.RK45DP64(g, cpu.m.copy())
    for _ in range(6):
        a = cpu.step()
        b = st.step()
        assert a == b
        assert st.time == pytest.approx(cpu.solver.time, rel=1e-12)
        assert st.dt == pytest.approx(cpu.solver.dt, rel=1e-9)
    assert np.abs(st.m.numpy() - cpu.m).max() < 1e-12


@pytest.mark.parametrize("openbc", [False, True])
def test_dmi_torque_and_field(openbc):
    """Exchange + interfacial DMI (dmi.cl) with per-region D, the boundary
    extrapolation and two empty cells, against the CPU oracle's FP64 variant."""
    regions, Ms, aex_r, Ku1, u, m0 = case()
    din = np.zeros(256)
    din[:4] = [3e-3, 2e-3, 3e-3, 1e-3]
    m0 = m0.copy()
    m0[:, 1, 4, 5] = 0.0
    m0[:, 0, 0, 3] = 0.0
    B_ext = (0.0, 0.01, 0.02)
    cpu = O.Simulation(N, CELL, Ms, 0.0, 0.05, dtype=np.float64, Ku1=Ku1, anisU=u, B_ext=B_ext, regions=regions,
                       Aex_regions=aex_r, Dind_regions=din, openbc=openbc)
    g = gpu64.System64(N, CELL, Ms, O.exch_lut(aex_r, dtype=np.float64), regions, 0.05,
                       kernel=O.newell_kernel(N, CELL), Ku1=Ku1, anisU=u, B_ext=B_ext, device="cpu",
                       dLUT=O.exch_lut(din, dtype=np.float64), openbc=openbc)
    cpu.set_m(m0)
    assert (cpu.m[:, 1, 4, 5] == 0).all()
    tau, B = cpu.torque(beff=True)
    m = torch.as_tensor(cpu.m)
    assert np.abs(g.beff(m).numpy() - B).max() <= 1e-12 * np.abs(B).max()
    assert np.abs(g.torque(m).numpy() - tau).max() <= 1e-12 * np.abs(tau).max()
