"""Ensembles: instances of several sizes and parameters advanced together
give bit-for-bit the trajectories each instance has when run alone with the
plain engine (the batched kernels share the single-instance arithmetic)."""
import numpy as np
import pytest

from tests import golden_pins as G

pytestmark = pytest.mark.gpu


def _inst(n, ms, aex, alpha, b, **kw):
    d = dict(N=(n, n, 1), cell=(4e-9, 4e-9, 3e-9), Msat=ms, Aex=aex, alpha=alpha, B_ext=b)
    d.update(kw)
    return d


@pytest.mark.parametrize("demag", [True, False])
def test_ensemble_matches_individual_runs(demag):
    from umagnus_b200 import engine
    insts = [_inst(32, 8e5, 1.3e-11, 0.1, (0.0, 0.0, 0.01)),
             _inst(48, 5e5, 7e-12, 0.3, (0.02, 0.0, 0.0)),        # 2n = 96: radix-3 passes
             _inst(32, 1.1e6, 1.9e-11, 0.02, (0.0, 0.05, 0.05)),  # same class as instance 0
             _inst(64, 6e5, 1.0e-11, 0.45, (0.0, 0.0, 0.0)),
             _inst(32, 9e5, 1.2e-11, 0.2, (0.01, 0.01, 0.0), Dind=1e-3, Ku1=3e4, anisU=(0, 0, 1))]
    ens = engine.Ensemble(insts, demag=demag)
    assert ens.classes() == 3
    ms = [G.random_unit(d["N"], 40 + k) for k, d in enumerate(insts)]
    for k, m in enumerate(ms):
        ens.set_m(k, m)
    T = 2e-11
    ens.run(T, chunk=2)
    for k, d in enumerate(insts):
        sim = engine.Simulation(d["N"], d["cell"], d["Msat"], d["Aex"], d["alpha"], Dind=d.get("Dind", 0.0),
                                Ku1=d.get("Ku1", 0.0), anisU=d.get("anisU", (0, 0, 1)), B_ext=d["B_ext"], demag=demag)
        sim.set_m(ms[k])
        sim.run(T)
        a, b = ens.state(k), sim.state()
        assert (a["nsteps"], a["nundone"]) == (b["nsteps"], b["nundone"]), (k, a, b)
        assert a["time"] == b["time"] and a["dt"] == b["dt"]
        np.testing.assert_array_equal(ens.get_m(k), sim.get_m().cpu().numpy())
        sim.free()
    ens.free()
