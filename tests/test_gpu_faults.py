"""Error paths of the bounded device waits, through the C-ABI.

Kernels that wait for a bulk (TMA) copy poll their mbarrier a bounded
number of times; when the poll gives up, pass C counts the timeout and the
engine's kernels set the simulation's device-side status (7).  These tests
plant those values from the host (umag_debug_plant_fault) -- nothing on the
GPU faults or waits -- and check that the host-side checks turn them into
errors: umag_demag_exec returns UMAG_E_TIMEOUT instead of a silently
unwritten field (the reference aborts on a failed kernel,
opencl/opencl.go:20-30), and the engine's run reports a solver failure.
"""
import numpy as np
import pytest

from tests import golden_pins as G

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

UMAG_E_SOLVER, UMAG_E_TIMEOUT = 6, 7


def test_demag_exec_reports_timed_out_copies():
    from umagnus_b200 import _lib
    from umagnus_b200 import opencl as cl
    cl.Init(0)
    L = _lib.load()
    N = (64, 64, 16)
    d = cl.NewNewellDemag(N, (0, 0, 0), (2e-9, 2e-9, 1e-9))
    m = torch.as_tensor(G.random_unit(N, 3)).cuda()
    B = torch.zeros_like(m)
    d.Exec(B, m, None, 8e5)
    ref = B.clone()
    try:
        _lib.check(L.umag_debug_plant_fault(None, 1))
        rc = L.umag_demag_exec(d._h, *[B[c].data_ptr() for c in range(3)], *[m[c].data_ptr() for c in range(3)],
                               None, None, 8e5)
        assert rc == UMAG_E_TIMEOUT
        assert b"timed out" in L.umag_last_error()
    finally:
        _lib.check(L.umag_debug_plant_fault(None, 0))
    B.zero_()
    d.Exec(B, m, None, 8e5)  # cleared: the next field is complete and correct again
    assert torch.equal(B, ref)
    d.Free()


def test_simulation_reports_a_planted_wait_failure():
    from umagnus_b200 import _lib, engine
    N = (32, 32, 4)
    sim = engine.Simulation(N, (2e-9, 2e-9, 2e-9), 8e5, 1.3e-11, 0.1, Dind=1e-3, B_ext=(0, 0, 0.01))
    sim.set_m(G.random_unit(N, 4))
    sim.run(2e-13)
    assert sim.state()["status"] == 0
    L = _lib.load()
    _lib.check(L.umag_debug_plant_fault(ctypes_ptr(sim._h), 7))
    with pytest.raises(_lib.UmagError, match="solver failure code 7"):
        sim.run(2e-13)
    st = sim.state()
    assert st["status"] == 7
    sim.free()


def ctypes_ptr(h):
    import ctypes
    return ctypes.c_void_p(h)
