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


def test_ensemble_is_deterministic_and_matches_every_instance():
    """Two runs of a 40-instance mixed ensemble are identical, and every
    instance equals its single run."""
    import bench
    from umagnus_b200 import engine
    insts = bench.ensemble_instances(count=40, seed=11)
    runs = []
    for _ in range(2):
        ens = engine.Ensemble([{k: v for k, v in d.items() if k != "m_seed"} for d in insts])
        for i, d in enumerate(insts):
            ens.set_m(i, bench.random_m(d["N"], d["m_seed"]))
        ens.run(5e-12, chunk=2)
        runs.append(([ens.state(i) for i in range(len(insts))], [ens.get_m(i) for i in range(len(insts))]))
        ens.free()
    for i in range(len(insts)):
        assert runs[0][0][i] == runs[1][0][i], i
        np.testing.assert_array_equal(runs[0][1][i], runs[1][1][i])
    for i, d in enumerate(insts):
        sim = engine.Simulation(d["N"], d["cell"], d["Msat"], d["Aex"], d["alpha"], B_ext=d["B_ext"])
        sim.set_m(bench.random_m(d["N"], d["m_seed"]))
        sim.run(5e-12)
        st = sim.state()
        assert (st["nsteps"], st["nundone"], st["time"], st["dt"]) == (
            runs[0][0][i]["nsteps"], runs[0][0][i]["nundone"], runs[0][0][i]["time"], runs[0][0][i]["dt"]), i
        np.testing.assert_array_equal(sim.get_m().cpu().numpy(), runs[0][1][i])
        sim.free()


def test_ensemble_error_against_fp64_oracle():
    """Two ensemble instances against the FP64 oracle (uMagNUS64 restated)
    after 20 ps of adaptive RK45DP: <m> within 1e-4, every cell within 1e-3
    (float32 state and FFT against FP64; the ensemble is bit-identical to
    the single-instance engine, so this is also the plain form's error)."""
    from oracle import oracle as O
    import bench
    from umagnus_b200 import engine
    insts = [dict(N=(32, 32, 1), cell=(4e-9, 4e-9, 3e-9), Msat=7e5, Aex=1.1e-11, alpha=0.2, B_ext=(0.03, 0.0, 0.04)),
             dict(N=(48, 48, 1), cell=(4e-9, 4e-9, 3e-9), Msat=1.0e6, Aex=1.6e-11, alpha=0.35, B_ext=(0.0, 0.05, 0.0))]
    ens = engine.Ensemble(insts)
    ms = [bench.random_m(d["N"], 100 + i) for i, d in enumerate(insts)]
    for i, m in enumerate(ms):
        ens.set_m(i, m)
    T = 2e-11
    ens.run(T)
    for i, d in enumerate(insts):
        orc = O.Simulation(d["N"], d["cell"], d["Msat"], d["Aex"], d["alpha"], dtype=np.float64, B_ext=d["B_ext"])
        orc.set_m(ms[i].astype(np.float64))
        orc.run(T)
        got = ens.get_m(i).astype(np.float64)
        want = orc.m.reshape(got.shape)
        assert np.max(np.abs(got - want)) < 1e-3
        assert np.max(np.abs(got.reshape(3, -1).mean(1) - want.reshape(3, -1).mean(1))) < 1e-4
    ens.free()


def test_ensemble_compaction_and_second_run():
    """Instances that finish early leave the batch (the running ones are
    compacted to its front and the class's graph recaptured); a second run
    brings every instance back.  Each instance still equals its single run
    after both runs, bit for bit, and ensemble indices keep naming the same
    instances."""
    import bench
    from umagnus_b200 import engine
    insts = bench.ensemble_instances(count=24, seed=23)
    # low damping on a few instances makes their step counts far larger
    for k in (1, 7, 12):
        insts[k]["alpha"] = 0.011
    ens = engine.Ensemble([{k: v for k, v in d.items() if k != "m_seed"} for d in insts])
    for i, d in enumerate(insts):
        ens.set_m(i, bench.random_m(d["N"], d["m_seed"]))
    ens.run(4e-12, chunk=1)
    first = [ens.state(i) for i in range(len(insts))]
    ens.run(3e-12, chunk=1)
    for i, d in enumerate(insts):
        sim = engine.Simulation(d["N"], d["cell"], d["Msat"], d["Aex"], d["alpha"], B_ext=d["B_ext"])
        sim.set_m(bench.random_m(d["N"], d["m_seed"]))
        sim.run(4e-12)
        s1 = sim.state()
        assert (s1["nsteps"], s1["time"], s1["dt"]) == (first[i]["nsteps"], first[i]["time"], first[i]["dt"]), i
        sim.run(3e-12)
        s2, e2 = sim.state(), ens.state(i)
        assert (s2["nsteps"], s2["nundone"], s2["time"], s2["dt"]) == (
            e2["nsteps"], e2["nundone"], e2["time"], e2["dt"]), i
        np.testing.assert_array_equal(sim.get_m().cpu().numpy(), ens.get_m(i))
        sim.free()
    ens.free()


def test_class_launch_shapes_change_nothing_but_speed():
    """Launch shapes set per class (as the ensemble autotuner does) leave
    every instance's trajectory bit for bit the same."""
    import bench
    from umagnus_b200 import engine
    insts = bench.ensemble_instances(count=12, seed=31)
    runs = []
    for shapes in (None, {"torque_block": [64, 2], "stage_threads": 128, "stage_waves": 2, "err_waves": 16}):
        ens = engine.Ensemble([{k: v for k, v in d.items() if k != "m_seed"} for d in insts])
        if shapes:
            for c in range(ens.classes()):
                ens.set_tuning(c, shapes)
                assert ens.get_tuning(c)["stage_threads"] == 128
        for i, d in enumerate(insts):
            ens.set_m(i, bench.random_m(d["N"], d["m_seed"]))
        ens.run(3e-12, chunk=2)
        runs.append(([ens.state(i) for i in range(len(insts))], [ens.get_m(i) for i in range(len(insts))]))
        ens.free()
    for i in range(len(insts)):
        assert runs[0][0][i] == runs[1][0][i], i
        np.testing.assert_array_equal(runs[0][1][i], runs[1][1][i])


def test_ensemble_autotune_chooses_and_caches(tmp_path):
    """The ensemble tuner gives every class valid shapes, stores them and
    applies the cached ones without timing the second time."""
    import bench
    from umagnus_b200 import engine
    insts = [d for d in bench.ensemble_instances(count=20, seed=3) if d["N"][0] in (32, 48)]
    clean = [{k: v for k, v in d.items() if k != "m_seed"} for d in insts]
    ens = engine.Ensemble(clean)
    cache = str(tmp_path / "tune.json")
    chosen, logs = ens.autotune(clean, cache_path=cache)
    assert set(chosen) == set(range(ens.classes())) and all(v is not None for v in logs.values())
    ens2 = engine.Ensemble(clean)
    chosen2, logs2 = ens2.autotune(clean, cache_path=cache)
    assert chosen2 == chosen and all(v is None for v in logs2.values())
    ens.free()
    ens2.free()


def _general_instances():
    """Instances the batched kernels do not serve: a region map with
    per-region exchange, Ms map and per-region applied field; a geometry
    mask (disc); periodic boundaries with interfacial DMI; a thermal field."""
    n = 32
    shape = (1, n, n)
    yy, xx = np.mgrid[0:n, 0:n]
    regions = ((xx >= n // 2).astype(np.uint8) + 2 * (yy >= n // 2).astype(np.uint8)).reshape(shape)
    ms_map = np.where(regions == 0, 8e5, 6e5).astype(np.float32)
    bext = np.zeros((256, 3), np.float32)
    bext[1] = (0.01, 0.0, 0.0)
    bext[3] = (0.0, 0.02, 0.0)
    disc = (((xx - n / 2 + 0.5) ** 2 + (yy - n / 2 + 0.5) ** 2) <= (n / 2 - 1) ** 2).astype(np.float32).reshape(shape)
    base = dict(N=(n, n, 1), cell=(4e-9, 4e-9, 3e-9), alpha=0.1)
    return [
        dict(base, Msat=ms_map, Aex=[1.3e-11, 1.0e-11, 1.5e-11, 1.2e-11], regions=regions, B_ext=bext),
        dict(base, Msat=8e5, Aex=1.3e-11, geom=disc, B_ext=(0.0, 0.0, 0.01)),
        dict(base, Msat=9e5, Aex=1.2e-11, Dind=1e-3, pbc=(2, 0, 0), B_ext=(0.01, 0.01, 0.0)),
        dict(base, Msat=8e5, Aex=1.3e-11, Temp=50.0, ThermSeed=5, B_ext=(0.0, 0.0, 0.02)),
    ]


def test_ensemble_general_instances_match_single_runs():
    """General instances (region maps, geometry, PBC, thermal field) run in
    an ensemble beside batched uniform ones; each ends bit for bit where the
    same Simulation run alone ends, and the batched instances still match
    theirs."""
    from umagnus_b200 import engine
    gen = _general_instances()
    uni = [_inst(32, 8e5, 1.3e-11, 0.1, (0.0, 0.0, 0.01)), _inst(32, 1.1e6, 1.9e-11, 0.02, (0.0, 0.05, 0.05))]
    insts = [uni[0], gen[0], gen[1], uni[1], gen[2], gen[3]]
    assert [engine.Ensemble.is_general(d) for d in insts] == [False, True, True, False, True, True]
    ens = engine.Ensemble(insts)
    assert ens.classes() == 5  # the two uniform films share one batch
    assert [ens.class_general(c) for c in range(5)] == [False, True, True, True, True]
    ms = [G.random_unit(d["N"], 70 + k) for k, d in enumerate(insts)]
    for k, m in enumerate(ms):
        ens.set_m(k, m)
    T = 2e-11
    ens.run(T, chunk=2)
    ens.run(T / 2, chunk=3)  # a second run continues every instance from its own time
    for k, d in enumerate(insts):
        sim = engine.Simulation(**d)
        sim.set_m(ms[k])
        sim.run(T)
        sim.run(T / 2)
        a, b = ens.state(k), sim.state()
        assert (a["nsteps"], a["nundone"]) == (b["nsteps"], b["nundone"]), (k, a, b)
        assert a["time"] == b["time"] and a["dt"] == b["dt"], (k, a, b)
        np.testing.assert_array_equal(ens.get_m(k), sim.get_m().cpu().numpy())
        sim.free()
    ens.free()


def test_ensemble_all_general_and_set_m_in_geometry():
    """An ensemble of general instances only; set_m keeps a geometry's empty
    cells at zero, as Simulation.set_m does."""
    from umagnus_b200 import engine
    gen = _general_instances()
    ens = engine.Ensemble([gen[1], gen[1]])
    assert ens.classes() == 2  # general instances never share a batch
    m = G.random_unit(gen[1]["N"], 3)
    ens.set_m(0, m)
    sim = engine.Simulation(**gen[1])
    sim.set_m(m)
    np.testing.assert_array_equal(ens.get_m(0), sim.get_m().cpu().numpy())
    assert np.all(ens.get_m(0)[:, gen[1]["geom"] == 0] == 0)
    sim.free()
    ens.free()


def test_ensemble_autotune_with_bench_records_and_general_instances(tmp_path):
    """The tuner takes the instance records as bench.py passes them (with
    their m_seed key) and skips general instances, which keep the
    single-simulation shapes."""
    import bench
    from umagnus_b200 import engine
    insts = [d for d in bench.ensemble_instances(count=12, seed=5) if d["N"][0] == 32][:3]
    assert insts
    gen = _general_instances()[1]
    clean = [{k: v for k, v in d.items() if k != "m_seed"} for d in insts] + [gen]
    ens = engine.Ensemble(clean)
    assert [ens.class_general(c) for c in range(ens.classes())] == [False, True]
    before = ens.get_tuning(1)
    chosen, logs = ens.autotune(insts + [gen], cache_path=str(tmp_path / "tune.json"))
    assert set(chosen) == {0} and logs[0] is not None
    assert ens.get_tuning(1) == before
    ens.free()
