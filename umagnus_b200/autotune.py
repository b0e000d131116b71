"""Autotuner for the launch shapes of the per-cell kernels of a Simulation
and of the batched classes of an Ensemble.

The tunables (umag_tuning in the C header) are the CTA shape of the field +
torque kernel and whether its stencils read TMA-loaded tiles (where the
mesh allows them) or global memory, the threads and CTAs-per-SM cap of the
stage sums, and the CTAs-per-SM cap of the error norms.  They change speed only: every cell's
arithmetic is the same and the reductions are maxima, so a trajectory is bit
for bit the same under every shape.  The FFT passes have no runtime shape:
their thread layout is fixed by the register FFT's line length at compile
time.

The search is coordinate descent (torque block first, timed on field +
torque evaluations; then the stage shape and the error-norm cap, timed on
whole steps from a saved state), each candidate timed with CUDA events on the
stream the library runs on.  Choices are cached in a JSON file keyed by the
GPU name, the mesh and the terms that change the kernels' instruction mix.
"""
import json
import os
import tempfile

DEFAULT = {"torque_block": [32, 8], "stage_threads": 256, "stage_waves": 8, "err_waves": 4, "torque_tma": 1}
STAGE_SHAPES = [(th, w) for th in (128, 256) for w in (2, 4, 8, 16)]
ERR_WAVES = [2, 4, 8, 16]


def torque_blocks(nx):
    """CTA shapes (x, y) for the torque kernel: x a multiple of 32 no wider
    than the mesh row rounded up to 32, 64 <= x*y <= 256."""
    wmax = max(32, (nx + 31) // 32 * 32)
    out = []
    for bx in (32, 64, 128, 256):
        if bx > wmax:
            continue
        for by in (1, 2, 4, 8):
            if 64 <= bx * by <= 256:
                out.append((bx, by))
    return out


def cache_key(device_name, N, features):
    """Key of one tuning: the GPU, the mesh and the feature string."""
    return f"{device_name}|{N[0]}x{N[1]}x{N[2]}|{features}"


def default_cache_path():
    return os.environ.get("UMAG_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "umagnus_b200", "tuning.json"))


def load_cache(path):
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(path, data):
    """Write atomically (a concurrent reader sees the old or the new file)."""
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=d, prefix=".tuning.")
    with os.fdopen(fd, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def search(measure, nx, tma_choices=(1, 0)):
    """Coordinate descent over the three tunables.  measure(kind, tuning) ->
    seconds, kind "torque" or "step"; returns (best tuning, {kind: timings})."""
    best = {k: (list(v) if isinstance(v, list) else v) for k, v in DEFAULT.items()}
    log = {"torque": {}, "stage": {}, "err": {}}
    for bx, by in torque_blocks(nx):
        for tma in tma_choices:
            t = dict(best, torque_block=[bx, by], torque_tma=tma)
            log["torque"][f"{bx}x{by}/{tma}"] = measure("torque", t)
    shape, tma = min(log["torque"], key=log["torque"].get).split("/")
    bx, by = (int(v) for v in shape.split("x"))
    best["torque_block"], best["torque_tma"] = [bx, by], int(tma)
    for th, w in STAGE_SHAPES:
        t = dict(best, stage_threads=th, stage_waves=w)
        log["stage"][f"{th}/{w}"] = measure("step", t)
    th, w = (int(v) for v in min(log["stage"], key=log["stage"].get).split("/"))
    best["stage_threads"], best["stage_waves"] = th, w
    for w in ERR_WAVES:
        log["err"][str(w)] = measure("step", dict(best, err_waves=w))
    best["err_waves"] = int(min(log["err"], key=log["err"].get))
    return best, log


def features(sim):
    p = sim.params
    return "demag={}{}|dmi={}|anis={}|regions={}".format(
        int(p.enable_demag), "b" if p.demag_kernel else "n", int(bool(p.dLUT or p.dbulkLUT)),
        int(bool(p.Ku1 or p.Ku1_mul or p.Kc1 or p.Kc1_mul)), int(bool(p.regions)))


def tune(sim, cache_path=None, evals=40, steps=16, use_cache=True):
    """Choose and apply the launch shapes of `sim` (an engine.Simulation on
    the GPU).  With use_cache, a cached choice for the same key is applied without
    timing; a new choice is stored.  Returns (tuning, timings or None)."""
    import torch

    cache_path = cache_path or default_cache_path()
    key = cache_key(torch.cuda.get_device_name(), sim.N, features(sim))
    cache = load_cache(cache_path) if use_cache else {}
    if key in cache:
        sim.set_tuning(cache[key])
        return sim.get_tuning(), None
    stream = torch.cuda.Stream()
    m0 = sim.get_m().clone()
    st0 = sim.state()
    previous = getattr(sim, "stream", None)  # the caller's stream, put back at the end
    sim.set_stream(stream)
    try:
        def measure(kind, t):
            sim.set_tuning(t)
            n = evals if kind == "torque" else steps
            run = sim.torque_evals if kind == "torque" else sim.steps
            best = float("inf")
            for _ in range(3):  # warm-up (graph capture) + two timed repeats
                if kind == "step":
                    sim.restore_m(m0)
                    sim.set_time(st0["time"], st0["dt"])
                with torch.cuda.stream(stream):
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    run(n)
                    b.record(stream)
                b.synchronize()
                best = min(best, a.elapsed_time(b) * 1e-3)
            return best

        best, log = search(measure, sim.N[0])
        sim.set_tuning(best)
    finally:
        sim.restore_m(m0)
        sim.set_time(st0["time"], st0["dt"])
        torch.cuda.synchronize()
        sim.set_stream(previous)
    if use_cache:
        cache = load_cache(cache_path)
        cache[key] = sim.get_tuning()
        save_cache(cache_path, cache)
    return sim.get_tuning(), log


def tune_ensemble(ens, instances, cache_path=None, use_cache=True, probe_size=8, replays=3):
    """Choose and apply the launch shapes of every class of `ens` (an
    engine.Ensemble made from `instances`).  Each class is timed on a probe
    ensemble of up to probe_size of its instances (fresh random states, a
    stop time no instance reaches, `replays` graph replays per candidate,
    wall clock around whole runs), so the real ensemble's state is never
    touched; the same coordinate descent as tune(), every kind timed on
    steps, no TMA tiles (a batch's torque kernel reads global memory).  With
    use_cache a cached choice is applied without timing.  Returns
    ({class: tuning}, {class: timings or None})."""
    import time

    import numpy as np
    import torch

    from .engine import Ensemble
    cache_path = cache_path or default_cache_path()
    cache = load_cache(cache_path) if use_cache else {}
    name = torch.cuda.get_device_name()
    chosen, logs = {}, {}
    strip = ("m_seed",)
    for cls in range(ens.classes()):
        if ens.class_general(cls):  # a general instance keeps the single-simulation shapes
            continue
        N, _ = ens.class_info(cls)
        members = [d for d in instances if tuple(int(v) for v in d["N"]) == tuple(N)
                   and not Ensemble.is_general({k: v for k, v in d.items() if k not in strip})]
        feats = "ens|dmi={}|anis={}".format(int(any(d.get("Dind", 0) for d in members)),
                                            int(any(d.get("Ku1", 0) or d.get("Ku2", 0) for d in members)))
        key = cache_key(name, N, feats)
        if key in cache:
            ens.set_tuning(cls, cache[key])
            chosen[cls], logs[cls] = ens.get_tuning(cls), None
            continue
        probe_insts = [{k: v for k, v in d.items() if k not in strip} for d in members[:probe_size]]
        probe = Ensemble(probe_insts)
        rng = np.random.default_rng(7)
        for i, d in enumerate(probe_insts):
            m = rng.standard_normal((3, d["N"][2], d["N"][1], d["N"][0]))
            probe.set_m(i, m / np.sqrt((m * m).sum(0)))
        try:
            def measure(kind, t):
                probe.set_tuning(0, t)
                best = float("inf")
                for rep in range(3):  # the first includes the graph capture
                    torch.cuda.synchronize()
                    a = time.perf_counter()
                    probe.run(1.0, chunk=replays, max_replays=replays)
                    torch.cuda.synchronize()
                    if rep:
                        best = min(best, time.perf_counter() - a)
                return best

            best, log = search(measure, N[0], tma_choices=(0,))
        finally:
            probe.free()
        best["torque_tma"] = 0
        ens.set_tuning(cls, best)
        chosen[cls], logs[cls] = ens.get_tuning(cls), log
        if use_cache:
            c = load_cache(cache_path)
            c[key] = chosen[cls]
            save_cache(cache_path, c)
    return chosen, logs
