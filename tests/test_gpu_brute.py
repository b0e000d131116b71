"""The brute-force demag kernel (mag/demagkernel.go:113-336) on the GPU:
identical float32 values to the oracle's restatement, the mumax3 regression
values of test/demagSmall.mx3, demagSmall3D.mx3 and demagcube.mx3, and an
engine torque with it against the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests import golden_pins as G

pytestmark = pytest.mark.gpu
MU0 = 4e-7 * np.pi


@pytest.mark.parametrize("N,cell", [((3, 4, 1), (1e-9, 2e-9, 0.5e-9)), ((3, 4, 2), (1e-9, 2e-9, 3e-9)),
                                    ((2, 2, 2), (1e-9, 1e-9, 1e-9)), ((7, 5, 3), (2e-9, 3e-9, 1e-9)),
                                    ((12, 9, 6), (4e-9, 4e-9, 2e-9))])
def test_kernel_equals_oracle(N, cell):
    from umagnus_b200 import opencl as cl
    d = cl.NewBruteDemag(N, (0, 0, 0), cell)
    got = d.kernel()
    want = O.brute_kernel(N, cell).astype(np.float64)
    np.testing.assert_array_equal(got, want)
    d.Free()


@pytest.mark.parametrize("N,cell,pbc", [((6, 4, 1), (1e-9, 2e-9, 1e-9), (2, 1, 0)),
                                         ((4, 4, 3), (2e-9, 2e-9, 1e-9), (0, 0, 2))])
def test_pbc_kernel_equals_oracle(N, cell, pbc):
    """Periodic images accumulated in float32 in the reference's loop order."""
    from umagnus_b200 import opencl as cl
    d = cl.NewBruteDemag(N, pbc, cell)
    got = d.kernel()
    want = O.brute_kernel(N, cell, pbc).astype(np.float64)
    np.testing.assert_array_equal(got, want)
    d.Free()


@pytest.mark.parametrize("N,cell,want,tol", [
    ((3, 4, 1), (1e-9, 2e-9, 0.5e-9), (-0.15768295526, -0.05676037073, -0.78447151184), 1e-6),  # demagSmall.mx3
    ((3, 4, 2), (1e-9, 2e-9, 3e-9), (-0.52710835138, -0.20121671756, -0.27112555503), 1e-6),   # demagSmall3D.mx3
    ((2, 2, 2), (1e-9, 1e-9, 1e-9), (-1 / 3, -1 / 3, -1 / 3), 5e-4),                              # demagcube.mx3
])
def test_regression_values(N, cell, want, tol):
    """B_demag.Average() of uniform m along x, y, z with Msat = 1/mu0."""
    from umagnus_b200 import opencl as cl
    d = cl.NewBruteDemag(N, (0, 0, 0), cell)
    B = torch.empty((3, N[2], N[1], N[0]), dtype=torch.float32, device="cuda")
    for i in range(3):
        m = torch.zeros_like(B)
        m[i] = 1.0
        d.Exec(B, m, None, float(np.float32(1 / MU0)))
        avg = B.reshape(3, -1).double().mean(dim=1).cpu().numpy()
        for j in range(3):
            assert abs(avg[j] - (want[i] if i == j else 0.0)) <= tol, (i, j, avg[j])
    d.Free()


def test_engine_torque_with_brute_kernel():
    from umagnus_b200 import engine
    N, cell = (24, 16, 4), (3e-9, 3e-9, 2e-9)
    kw = dict(Dind=1e-3, Ku1=2e5, anisU=(0, 0, 1), B_ext=(0.01, 0.0, 0.02))
    sim = engine.Simulation(N, cell, 8e5, 1.3e-11, 0.1, demag_kernel="brute", **kw)
    m = G.random_unit(N, 9)
    sim.set_m(m)
    tau = sim.torque().cpu().numpy()
    Kf, _ = O.kernel_spectrum(O.brute_kernel(N, cell).astype(np.float64))
    orc = O.Simulation(N, cell, 8e5, 1.3e-11, 0.1, kernel=Kf, **kw)
    orc.set_m(sim.get_m().cpu().numpy())
    want = orc.torque()
    assert np.max(np.abs(tau - want)) <= 1e-5 * np.abs(want).max()
    sim.free()
