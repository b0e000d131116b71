"""Parity at the benchmarked sizes, against the FP64 oracle.

The benchmark times the compile-time-planned demag passes of the
256x256x16 multilayer (k_reg_a<256,32>, k_reg_b<512,4>, k_reg_c<256,32>) and
the precision workload runs those of 512x512x32 (k_reg_a<512,64>,
k_reg_b<1024,.>, k_reg_c<512,64>).  These tests run exactly those
instantiations through the engine and the C-ABI and compare them with the
FP64 restatement of the path on the GPU (oracle/gpu64.py: uMagNUS64's
semantics, pinned to the CPU oracle by tests/test_fp64_oracle.py), whose
Newell tensor comes from the CPU oracle (oracle/orc_newell.c), so nothing
of the product is in the reference values.

Tolerances, as the path promises (1e-5 relative per cell against FP64):
|dB| <= 1e-5 max|B| and |dtau| <= 1e-5 max|tau| for one evaluation; after a
few RK45DP steps the same accept decisions, m within 1e-5 per cell and the
accepted dt within 1e-3 relative (dt follows the error estimate, a ratio of
small differences).
"""
import numpy as np
import pytest

from oracle import gpu64
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-5


def _multilayer():
    import bench
    c = bench.CONFIG
    return c, bench.random_m(c["N"], c["seed"])


def _fp64_multilayer(c):
    N = c["N"]
    return gpu64.System64(N, c["cell"], c["Ms"], O.exch_lut(np.full(256, c["Aex"]), dtype=np.float64),
                          np.zeros(N[::-1], np.uint8), c["alpha"], kernel=O.newell_kernel(N, c["cell"]),
                          Ku1=c["Ku1"], anisU=c["anisU"], B_ext=c["B_ext"],
                          dLUT=O.exch_lut(np.full(256, c["Dind"]), dtype=np.float64))


def _sim(c):
    from umagnus_b200 import engine
    return engine.Simulation(c["N"], c["cell"], c["Ms"], c["Aex"], c["alpha"], Dind=c["Dind"], Ku1=c["Ku1"],
                             anisU=c["anisU"], B_ext=c["B_ext"])


def _rel(a, b):
    """max |a - b| per cell (vector norm) over max |b|, and the RMS ratio."""
    d = torch.sqrt(((a.double() - b) ** 2).sum(0))
    n = torch.sqrt((b ** 2).sum(0))
    return float(d.max() / n.max()), float(torch.sqrt((d ** 2).mean() / (n ** 2).mean()))


def test_multilayer_field_and_torque_match_fp64():
    c, m0 = _multilayer()
    sim = _sim(c)
    sim.set_m(m0)
    tau, B = sim.torque(beff=True)
    m = sim.get_m().reshape((3,) + sim.shape).double()
    sys64 = _fp64_multilayer(c)
    B64 = sys64.beff(m)
    t64 = sys64.torque(m, B64)
    eB, _ = _rel(B.reshape(B64.shape), B64)
    et, _ = _rel(tau.reshape(t64.shape), t64)
    sim.free()
    assert eB <= TOL, eB
    assert et <= TOL, et


def test_multilayer_rk45dp_steps_match_fp64():
    c, m0 = _multilayer()
    sim = _sim(c)
    sim.set_m(m0)
    sys64 = _fp64_multilayer(c)
    st64 = gpu64.RK45DP64(sys64, sim.get_m().reshape((3,) + sim.shape).double().cpu().numpy())
    prev = sim.state()
    for i in range(5):
        sim.steps(1)
        s = sim.state()
        t0 = st64.time
        acc64 = st64.step()
        assert (s["nsteps"] > prev["nsteps"]) == acc64, i
        if acc64:
            d32, d64 = s["time"] - prev["time"], st64.time - t0
            assert abs(d32 - d64) <= 1e-3 * d64, (i, d32, d64)
        prev = s
    m = sim.get_m().reshape((3,) + sim.shape).double()
    sim.free()
    assert float((m - st64.m).abs().max()) <= TOL


def test_demag_512x512x32_matches_fp64():
    from umagnus_b200 import opencl as cl
    cl.Init(0)
    N, cell, Ms = (512, 512, 32), (2e-9, 2e-9, 2e-9), 9e5
    rng = np.random.default_rng(31)
    m = rng.standard_normal((3, N[2], N[1], N[0]))
    m = (m / np.sqrt((m * m).sum(0))).astype(np.float32)
    d = cl.NewNewellDemag(N, (0, 0, 0), cell)
    mt = torch.as_tensor(m).cuda()
    B = torch.empty_like(mt)
    d.Exec(B, mt, None, Ms)
    d.Free()
    sys64 = gpu64.System64(N, cell, Ms, np.zeros(32896), np.zeros(N[::-1], np.uint8), 0.1,
                           kernel=O.newell_kernel(N, cell))
    B64 = sys64.demag_field(mt.double())
    del sys64
    e, _ = _rel(B, B64)
    assert e <= TOL, e


def test_precision_workload_field_matches_fp64():
    """The 512x512x32 precision workload (64 Voronoi grains, two grain
    classes of Ms and Aex, a random easy axis per grain): B_eff and tau of m0
    through the engine (region LUTs, per-cell maps) against FP64."""
    import bench
    pb = bench.precision_problem((512, 512, 32))
    from umagnus_b200 import engine
    N = pb["N"]
    sim = engine.Simulation(N, pb["cell"], Msat=pb["Ms"], Aex=pb["aex_r"], alpha=pb["alpha"], Ku1=pb["Ku1"],
                            anisU=pb["u"], regions=pb["regions"])
    sim.set_m(pb["m0"])
    tau, B = sim.torque(beff=True)
    m = sim.get_m().reshape((3,) + sim.shape).double()
    sys64 = gpu64.System64(N, pb["cell"], pb["Ms"].astype(np.float64), O.exch_lut(pb["aex_r"], dtype=np.float64),
                           pb["regions"], pb["alpha"], kernel=O.newell_kernel(N, pb["cell"]), Ku1=pb["Ku1"],
                           anisU=pb["u"].astype(np.float64))
    B64 = sys64.beff(m)
    t64 = sys64.torque(m, B64)
    sim.free()
    eB, _ = _rel(B.reshape(B64.shape), B64)
    et, _ = _rel(tau.reshape(t64.shape), t64)
    assert eB <= TOL, eB
    assert et <= TOL, et
