"""The CPU reference arm of bench.py (reference kernels on host threads +
scipy FFT + numpy RK45DP controller) agrees with the oracle's engine."""
import numpy as np
import pytest

from oracle import clref
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not clref.available(), reason="oracle/_ref/libclref.so not built")

CFG = dict(cell=(2e-9, 2e-9, 1e-9), Ms=1.1e6, Aex=1.6e-11, alpha=0.3, Dind=3e-3, Ku1=5e5, anisU=(0.0, 0.0, 1.0),
           B_ext=(0.0, 0.0, 0.05))


def _pair(N, threads):
    from oracle.ref_arm import RefRK45
    c = CFG
    o = O.Simulation(N, c["cell"], c["Ms"], c["Aex"], c["alpha"], Dind=c["Dind"], Ku1=c["Ku1"], anisU=c["anisU"],
                     B_ext=c["B_ext"])
    r = RefRK45(N, c["cell"], c["Ms"], c["Aex"], c["alpha"], c["Dind"], c["Ku1"], c["anisU"], c["B_ext"],
                threads=threads, Kf=o.Kf)
    rng = np.random.default_rng(5)
    m = rng.standard_normal((3, N[2], N[1], N[0]))
    m = (m / np.sqrt((m * m).sum(0))).astype(np.float32)
    o.set_m(m)
    r.set_m(o.m)
    return o, r


@pytest.mark.parametrize("threads", [1, 3])
def test_ref_arm_torque_matches_oracle(threads):
    o, r = _pair((32, 24, 4), threads)
    want = o.torque()
    got = np.zeros_like(want)
    r.torque(got, r.m)
    # the FFTs differ (scipy vs the oracle's own); the local terms are the
    # same reference kernels, so agreement is to float32 FFT rounding
    assert np.max(np.abs(got - want)) <= 1e-5 * np.abs(want).max()


def test_ref_arm_steps_match_oracle():
    o, r = _pair((16, 16, 2), 2)
    for _ in range(4):
        assert o.step() == r.step()
    assert abs(o.solver.time - r.time) <= 1e-6 * o.solver.time
    assert np.max(np.abs(o.m - r.m)) <= 1e-4
