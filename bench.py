"""Benchmark: RK45DP cell-updates/s of the 256x256x16 multilayer on B200.

Workload (the multilayer configuration): 256x256x16 cells of 2x2x1 nm, Ms
1.1e6 A/m, Aex 1.6e-11 J/m, interfacial D 3e-3 J/m^2, Ku1 5e5 J/m^3 along z,
alpha 0.3, B_ext (0, 0, 50 mT), Newell demag, float32, initial m i.i.d.
random unit vectors from a seed.  A "step" is one RK45DP step attempt
(6 field + torque evaluations, the stage sums, the fused error norms and the
device step controller); `value` counts accepted steps only.

Timing: W warm-up steps, then K steps between CUDA events on the stream the
library launches on, inside a barrier + synchronize on both sides; max over
ranks.  The device working set (state, 7 stage buffers, spectrum, kernel,
~0.2 GB) exceeds the 126 MB L2, so no flush is needed between steps.
Multi-GPU: the plain path does not shard (the demag convolution is a global
FFT), so N GPUs run N independent replicas ("replicas only").

--impl reference times the reference's implementation of the path on the
host cores: the reference's own OpenCL C kernels compiled for the host
(oracle/_ref) and spread over all host threads, scipy.fft (multi-threaded)
in place of the reference's vendored VkFFT (which needs an OpenCL device),
the RK45DP stepper and controller restated in numpy (oracle/ref_arm.py).

Accuracy: outside every timed region, B_eff and the torque of the seeded
m0 from the engine are compared with the FP64 oracle (oracle/gpu64.py, the
checker; its Newell tensor comes from the CPU oracle) and the line carries
the error (`error_vs_fp64`).  A CPU step takes seconds, so that arm times whole
steps until --steps or --ref-budget seconds, whichever comes first.
"""
import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIG = dict(N=(256, 256, 16), cell=(2e-9, 2e-9, 1e-9), Ms=1.1e6, Aex=1.6e-11, Dind=3e-3, Ku1=5e5,
              anisU=(0.0, 0.0, 1.0), alpha=0.3, B_ext=(0.0, 0.0, 0.05), seed=2)
METRIC = "RK45DP cell-updates/s (256x256x16 multilayer, FP32, Newell demag)"
UNIT = "cell-updates/s"
# dram__bytes_read.sum + dram__bytes_write.sum of one k_reg_b<512,4> launch on
# this workload (79,939,328 + 4,860,160 B), from one ncu --set full capture of
# that launch with packed FP32 butterflies and staged twiddle tables (cold
# cache: ncu flushes the caches between its passes)
TRAFFIC_B = 84799488
TRAFFIC_B_SOURCE = ("ncu capture of k_reg_b<512,4>, packed FP32 butterflies + staged twiddle tables "
                    "(profiles/k_reg_b_multilayer_256x256x16.md)")


def alg_bytes_per_eval(N):
    """Algorithmic HBM bytes of one field + torque evaluation:
    24N (read m, write tau) + 4*nK*K (Fourier kernel) + 48*S (one write + read
    of the 3-component half spectrum)."""
    Nx, Ny, Nz = N
    Px, Py = 2 * Nx, 2 * Ny
    Pz = 2 * Nz if Nz > 5 else 2 * Nz - 1
    S = (Px // 2 + 1) * Py * Pz
    K = (Px // 2 + 1) * (Py // 2 + 1) * (Pz // 2 + 1)
    nK = 4 if Nz == 1 else 6
    n = Nx * Ny * Nz
    return 24 * n + 4 * nK * K + 48 * S


def alg_bytes_per_pass(N):
    """Algorithmic HBM bytes of the three demag passes (uniform Ms, no vol):
    A reads m (12n) and writes the 3-component spectrum (stored rows y < Ny
    only: Ssp = 3*8*(Px/2+1)*Ny*Pz); B reads and writes it and reads the
    kernel (4*nK*K); C reads it and writes B (12n)."""
    Nx, Ny, Nz = N
    Px, Py = 2 * Nx, 2 * Ny
    Pz = 2 * Nz if Nz > 5 else 2 * Nz - 1
    Ssp = 3 * 8 * (Px // 2 + 1) * Ny * Pz
    K = (Px // 2 + 1) * (Py // 2 + 1) * (Pz // 2 + 1)
    nK = 4 if Nz == 1 else 6
    n = Nx * Ny * Nz
    return {"A": 12 * n + Ssp, "B": 2 * Ssp + 4 * nK * K, "C": Ssp + 12 * n}


def time_passes(N, cell, Ms, stream, reps=50):
    """Per-launch device time of each demag pass (CUDA events on the stream
    the passes are queued on), after 5 untimed rounds."""
    import torch
    from umagnus_b200 import opencl as cl
    d = cl.NewNewellDemag(N, (0, 0, 0), cell)
    m = torch.from_numpy(random_m(N, 7)).cuda()
    B = torch.empty_like(m)
    out = {}
    try:
        for _ in range(5):
            for p in range(3):
                d.ExecPass(p, B, m, None, Ms)
        for p, name in enumerate("ABC"):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                d.ExecPass(p, B, m, None, Ms)
            e1.record(stream)
            e1.synchronize()
            out[name] = e0.elapsed_time(e1) / reps
    finally:
        d.Free()
    return out


def random_m(N, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((3, N[2], N[1], N[0]))
    v /= np.sqrt((v * v).sum(axis=0))
    return v.astype(np.float32)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML every
    ~2 ms on a background thread during the timed region (read-only queries)."""

    REASONS = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown")]

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.samples = []
        self.max_mhz = None
        self.error = None
        self._stop = threading.Event()
        self._t = None

    def _handle(self, nv):
        import torch
        p = torch.cuda.get_device_properties(self.cuda_index)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        return nv.nvmlDeviceGetHandleByPciBusId(bus)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            self._sample()
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception as e:  # no NVML: report unsampled
            self.error = f"{type(e).__name__}: {e}"
        return self

    def _sample(self):
        nv = self.nv
        mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
        reasons = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
        self.samples.append((mhz, reasons))

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception as e:
                self.error = f"{type(e).__name__}: {e}"
                return
            time.sleep(0.002)

    def __exit__(self, *a):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0,
                    "error": self.error}
        reasons = set()
        for _, bits in self.samples:
            for name, attr in self.REASONS:
                if bits & int(getattr(self.nv, attr, 0)):
                    reasons.add(name)
        mhz = [s[0] for s in self.samples]
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": self.max_mhz, "reasons": sorted(reasons),
                "samples": len(mhz), "source": "nvml"}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU arm
def make_ref(config):
    """The reference's path on host cores (oracle/ref_arm.py); the Newell
    kernel setup (FP64, one thread) is not part of any timed region."""
    from oracle.ref_arm import RefRK45
    c = config
    r = RefRK45(c["N"], c["cell"], c["Ms"], c["Aex"], c["alpha"], c["Dind"], c["Ku1"], c["anisU"], c["B_ext"])
    r.set_m(random_m(c["N"], c["seed"]))
    return r


def time_ref(r, max_steps, budget_s):
    """Time whole RK45DP step attempts until max_steps or budget_s is spent
    (at least one); returns (seconds, attempts, accepted)."""
    acc0 = r.nsteps
    t0 = time.perf_counter()
    n = 0
    while n < max(1, max_steps):
        r.step()
        n += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    return time.perf_counter() - t0, n, r.nsteps - acc0


def cpu_baseline(config, budget_s=12.0):
    """Bounded sample of the workload on the host cores: the reference's own
    kernels (oracle/_ref, host threads) + scipy FFT, one warm-up step, then
    whole RK45DP steps for about budget_s seconds."""
    from oracle import clref
    if not clref.available():
        raise RuntimeError("oracle/_ref/libclref.so is not built (run __graft_entry__.build())")
    r = make_ref(config)
    r.step()
    t, n, acc = time_ref(r, 10 ** 6, budget_s)
    ncell = r.n
    return {"value": acc * ncell / t, "unit": UNIT, "cores": r.threads, "kind": "reference",
            "sample": (f"{n} RK45DP steps ({acc} accepted) of the full 256x256x16 workload in {t:.1f} s after one "
                       f"warm-up step: reference OpenCL C kernels compiled for the host on {r.threads} threads, "
                       "scipy.fft for the reference's VkFFT; Newell kernel setup excluded")}


# ------------------------------------------------------------------ accuracy
def error_vs_fp64(sim, m0, cfg):
    """B_eff and the torque of m0 from the engine (the kernels the benchmark
    times) against the FP64 oracle (oracle/gpu64.py with the CPU oracle's
    Newell tensor): max and RMS of |dB| / max|B|, |dtau| / max|tau|.  The
    oracle is the checker here; this runs after every timed region."""
    import torch
    from oracle import gpu64
    from oracle import oracle as O
    N = cfg["N"]
    sim.set_m(m0)
    tau, B = sim.torque(beff=True)
    m = sim.get_m().reshape((3,) + sim.shape).double()
    sys64 = gpu64.System64(N, cfg["cell"], cfg["Ms"], O.exch_lut(np.full(256, cfg["Aex"]), dtype=np.float64),
                           np.zeros(N[::-1], np.uint8), cfg["alpha"], kernel=O.newell_kernel(N, cfg["cell"]),
                           Ku1=cfg["Ku1"], anisU=cfg["anisU"], B_ext=cfg["B_ext"],
                           dLUT=O.exch_lut(np.full(256, cfg["Dind"]), dtype=np.float64))
    B64 = sys64.beff(m)
    t64 = sys64.torque(m, B64)
    del sys64

    def rel(a, b):
        d = torch.sqrt(((a.reshape(b.shape).double() - b) ** 2).sum(0))
        n = torch.sqrt((b ** 2).sum(0))
        return {"max_rel_to_max": float(d.max() / n.max()),
                "rms_rel_to_rms": float(torch.sqrt((d ** 2).mean() / (n ** 2).mean()))}

    out = {"B_eff": rel(B, B64), "torque": rel(tau, t64), "tolerance": 1e-5,
           "what": "one field + torque evaluation of the seeded m0 against the FP64 oracle"}
    out["within_tolerance"] = out["B_eff"]["max_rel_to_max"] <= 1e-5 and out["torque"]["max_rel_to_max"] <= 1e-5
    return out


# ------------------------------------------------------------------ GPU arm
def combine_ranks(times, counts, dist=None):
    """The replicas' figures as one job: the slowest rank's time for each
    timing (max over ranks) and the steps all ranks took (sum), so that the
    whole-job throughput is every rank's cell-updates over the slowest
    rank's time.  Every rank calls it; tensors on the process group's
    device."""
    if dist is not None:
        dist.all_reduce(times, op=dist.ReduceOp.MAX)
        dist.all_reduce(counts, op=dist.ReduceOp.SUM)
    return times.tolist(), counts.tolist()


def run_ours(args, rank, world, local_rank):
    import torch
    from umagnus_b200 import engine

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod
    cfg = CONFIG
    N = cfg["N"]
    ncell = N[0] * N[1] * N[2]
    sim = engine.Simulation(N, cfg["cell"], cfg["Ms"], cfg["Aex"], cfg["alpha"], Dind=cfg["Dind"], Ku1=cfg["Ku1"],
                            anisU=cfg["anisU"], B_ext=cfg["B_ext"], device=local_rank)
    m0 = random_m(N, cfg["seed"] + rank)
    sim.set_m(m0)
    # launch shapes of the per-cell kernels for this mesh on this GPU (the
    # search restores m and the time; results do not depend on the shapes)
    tuning = sim.get_tuning() if args.no_autotune else sim.autotune()[0]
    stream = torch.cuda.Stream()
    sim.set_stream(stream)
    graph_steps = 16
    sim.use_graph(True, graph_steps)
    # warm-up: W steps, then one replay of each CUDA graph the timed region
    # uses (graph_steps steps and the one-step remainder), so that capturing
    # and instantiating them is not timed
    warm = max(args.warmup, 3)
    sim.steps(warm)
    sim.steps(graph_steps)
    sim.steps(1)
    warm += graph_steps + 1
    stream.synchronize()
    st0 = sim.state()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        sim.steps(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    st1 = sim.state()
    acc = st1["nsteps"] - st0["nsteps"]
    rej = st1["nundone"] - st0["nundone"]
    if st1["status"] != 0:
        raise RuntimeError(f"solver failure {st1}")
    # field-evaluation roofline: time E evaluations alone on the same stream
    E = 60
    sim.torque_evals(5)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.torque_evals(E)
    e1.record(stream)
    e1.synchronize()
    ms_eval = e0.elapsed_time(e1) / E
    ms_pass = time_passes(N, cfg["cell"], cfg["Ms"], stream)
    # end-to-end through the public API with host buffers
    host_m = torch.from_numpy(m0).pin_memory()
    host_out = torch.empty_like(host_m).pin_memory()
    dev_m = torch.empty_like(host_m, device="cuda")
    dev_out = torch.empty_like(dev_m)
    # one untimed pass of the copies (first-use costs of the pinned buffers
    # and the transfer path are not per-run work)
    dev_m.copy_(host_m, non_blocking=True)
    sim.get_m(out=dev_out)
    host_out.copy_(dev_out)
    torch.cuda.synchronize()
    t_e0 = time.perf_counter()
    dev_m.copy_(host_m, non_blocking=True)
    sim.set_m(dev_m)
    # the same step count as the device-timed region: chunks of graph_steps
    # and the remainder, with a solver-state read-back after each chunk
    steps_e2e = args.steps
    s_before = sim.state()
    chunks, left = 0, steps_e2e
    while left > 0:
        n = min(graph_steps, left)
        sim.steps(n)
        s_now = sim.state()  # D2H of the solver state after every chunk
        left -= n
        chunks += 1
    out = sim.get_m(out=dev_out)
    host_out.copy_(out)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t_e0
    acc_e2e = s_now["nsteps"] - s_before["nsteps"]
    bytes_state = 88
    # accuracy of the timed path (checker, outside every timed region)
    err64 = error_vs_fp64(sim, m0, cfg) if rank == 0 else None
    (ms_max, ms_eval_max, t_e2e_max), (acc_tot, acc_e2e_tot) = combine_ranks(
        torch.tensor([ms, ms_eval, t_e2e], dtype=torch.float64, device="cuda"),
        torch.tensor([acc, acc_e2e], dtype=torch.float64, device="cuda"), dist)
    result = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        b_eval = alg_bytes_per_eval(N)
        bp = alg_bytes_per_pass(N)
        achieved = b_eval / (ms_eval_max * 1e-3) / 1e9
        value = acc_tot * ncell / (ms_max * 1e-3)
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random m)",
            "config": {"workload": "multilayer 256x256x16 cells 2x2x1 nm, DMI + uniaxial + Zeeman + Newell demag, "
                                   "RK45DP adaptive, MaxErr 1e-5",
                       "cells": ncell, "accepted_steps": int(acc_tot), "rejected_steps": int(rej),
                       "l2": "working set ~0.2 GB > 126 MB L2, no flush", "parallelism": f"replicas x{world}",
                       "graph_steps": graph_steps, "warmup_steps_done": warm, "launch_shapes": tuning,
                       "autotuned": not args.no_autotune},
            "roofline": {"bound": "hbm", "kernel": f"k_reg_b (demag pass B: y FFT, kernel multiply, inverse y)",
                         "achieved": bp["B"] / (ms_pass["B"] * 1e-3) / 1e9, "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": bp["B"] / (ms_pass["B"] * 1e-3) / 1e9 / peak,
                         "traffic": TRAFFIC_B, "traffic_source": TRAFFIC_B_SOURCE,
                         "alg_bytes_per_launch": bp["B"], "ms_per_launch": ms_pass["B"],
                         "passes": {k: {"ms": ms_pass[k], "alg_bytes": bp[k],
                                        "gbs": bp[k] / (ms_pass[k] * 1e-3) / 1e9} for k in "ABC"},
                         "field_eval": {"ms": ms_eval_max, "alg_bytes": b_eval, "gbs": achieved,
                                        "frac": achieved / peak,
                                        "what": "demag passes A,B,C + fused local field/torque kernel"}},
            "e2e": {"value": acc_e2e_tot * ncell / t_e2e_max, "unit": UNIT,
                    "h2d_bytes_per_step": (12 * ncell) / steps_e2e,
                    "d2h_bytes_per_step": (12 * ncell + bytes_state * chunks) / steps_e2e,
                    "steps": steps_e2e,
                    "how": "pinned host m -> device, set_m, the same step count as the timed region in graph "
                           "chunks of 16 (and the remainder) with a solver-state read-back per chunk, final m -> "
                           "pinned host; wall clock"},
            "gpu_launches": sim.launches_per_step() * args.steps,
            "clocks": clk.summary(),
            "error_vs_fp64": err64,
        }
    sim.free()
    return result


# ------------------------------------------------------------------ ensemble workload
ENS_SIZES = (32, 48, 64, 96, 128)
ENS_CELL = (4e-9, 4e-9, 3e-9)


def ensemble_instances(count=256, seed=5):
    """The 256-instance thin-film ensemble: n x n x 1 films, n uniform in
    {32, 48, 64, 96, 128}, 4x4x3 nm cells; Ms U[4e5, 1.2e6] A/m, Aex
    U[5e-12, 2e-11] J/m, alpha U[0.01, 0.5], B_ext of random direction and
    magnitude U[0, 100] mT; m0 random unit vectors (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(ENS_SIZES))
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        b = d * rng.uniform(0.0, 0.1)
        out.append(dict(N=(n, n, 1), cell=ENS_CELL, Msat=float(rng.uniform(4e5, 1.2e6)),
                        Aex=float(rng.uniform(5e-12, 2e-11)), alpha=float(rng.uniform(0.01, 0.5)),
                        B_ext=tuple(float(x) for x in b), m_seed=int(rng.integers(1 << 31))))
    return out


def partition_instances(insts, world):
    """Instances over ranks, greedy longest-processing-time: largest meshes
    first, each to the rank with the fewest cells so far (instances are
    independent: no collective during the run)."""
    order = sorted(range(len(insts)), key=lambda i: -insts[i]["N"][0] * insts[i]["N"][1])
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += insts[i]["N"][0] * insts[i]["N"][1]
    return [sorted(x) for x in out]


def alg_bytes_per_step(N):
    """Algorithmic HBM bytes of one accepted RK45DP step: 6 field + torque
    evaluations and 480 bytes per cell of stage sums, error combination and
    m0 backup (40 vector accesses of 12 bytes; FSAL by pointer swap)."""
    return 6 * alg_bytes_per_eval(N) + 480 * N[0] * N[1] * N[2]


def ensemble_shard(insts_all, T, rank, world, dist, make_ensemble, device="cuda"):
    """This rank's share of the instances (partition_instances), run as one
    batched ensemble to simulated time T with no collective during the run;
    then one max (time) and one sum (instances, cell-updates, algorithmic
    bytes) over the ranks (combine_ranks).  make_ensemble(instances) returns
    an object with set_m(i, m), run(T, chunk), state(i) and free().  Returns
    (slowest rank's seconds, cell-updates, instances, bytes, this rank's
    instances, their final states)."""
    import torch
    mine = partition_instances(insts_all, world)[rank]
    insts = [insts_all[i] for i in mine]
    ens = make_ensemble(insts)
    for i, d in enumerate(insts):
        ens.set_m(i, random_m(d["N"], d["m_seed"]))
    sync = torch.cuda.synchronize if device == "cuda" else (lambda: None)
    sync()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    ens.run(T, chunk=8)
    sync()
    t_local = time.perf_counter() - t0
    states = [ens.state(i) for i in range(len(insts))]
    ens.free()
    acc = np.array([s["nsteps"] for s in states], float)
    ncell = [d["N"][0] * d["N"][1] for d in insts]
    alg = float(sum(a * alg_bytes_per_step(d["N"]) for a, d in zip(acc, insts)))
    (t_batch,), (cells_steps, n_done, alg_tot) = combine_ranks(
        torch.tensor([t_local], dtype=torch.float64, device=device),
        torch.tensor([float(np.dot(acc, ncell)), float(len(insts)), alg], dtype=torch.float64, device=device), dist)
    return t_batch, cells_steps, n_done, alg_tot, insts, states


def ensemble_measure(args, rank=0, world=1, dist=None, local_rank=0, plain=True, fp64_check=True):
    """The 256-instance ensemble: batched run of this rank's share
    (partition_instances; no collective during the run) to t = args.ens_time
    per instance, the job's time being the slowest rank's.  On rank 0 (plain
    = True) the plain engine one instance at a time on a per-size sample
    (args.ens_plain_sample of each size, extrapolated; every sampled
    instance must take exactly the batched instance's steps), and the error
    against the FP64 oracle of two sampled instances run to
    args.ens_check_time.  Returns the summary dict on rank 0, else None."""
    import torch
    from umagnus_b200 import engine
    insts_all = ensemble_instances()
    T = args.ens_time

    tunings = {}

    def make(ins):
        e = engine.Ensemble([{k: v for k, v in d.items() if k != "m_seed"} for d in ins], device=local_rank)
        # launch shapes of each class's batched kernels (speed only), before timing
        chosen, _ = e.autotune(ins)
        tunings.update({"x".join(str(v) for v in e.class_info(c)[0]): t for c, t in chosen.items()})
        return e

    t_batch, cells_steps, n_done, alg_tot, insts, states = ensemble_shard(insts_all, T, rank, world, dist, make)
    ncell = [d["N"][0] * d["N"][1] for d in insts]
    acc = np.array([s["nsteps"] for s in states], float)
    if rank != 0:
        return None
    peak, peak_kind = measured_peak()
    out = {"instances": int(n_done), "ranks": world, "simulated_time_s": T,
           "batched": {"seconds": t_batch, "instances_per_s": n_done / t_batch,
                       "cell_updates_per_s": cells_steps / t_batch,
                       "hbm": {"alg_bytes": alg_tot, "gbs": alg_tot / t_batch / 1e9, "peak": peak,
                               "peak_source": peak_kind, "frac": alg_tot / t_batch / 1e9 / peak,
                               "what": "sum over instances of accepted steps x (6 B_eval + 480 N) / wall time"},
                       "accepted_steps_rank0": {"total": int(acc.sum()), "min": int(acc.min()), "max": int(acc.max())},
                       "launch_shapes_rank0": tunings}}
    if not plain or world != 1:
        return out
    per_size = {}
    for n in ENS_SIZES:
        idx = [i for i, d in enumerate(insts) if d["N"][0] == n][: args.ens_plain_sample]
        ts = []
        for i in idx:
            d = insts[i]
            sim = engine.Simulation(d["N"], d["cell"], d["Msat"], d["Aex"], d["alpha"], B_ext=d["B_ext"])
            sim.set_m(random_m(d["N"], d["m_seed"]))
            torch.cuda.synchronize()
            a = time.perf_counter()
            sim.run(T)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - a)
            st = sim.state()
            assert st["nsteps"] == states[i]["nsteps"], "plain and batched trajectories differ"
            sim.free()
        per_size[n] = (float(np.mean(ts)), len(idx))
    t_plain = sum(per_size[d["N"][0]][0] for d in insts)
    out["plain"] = {"seconds_extrapolated": t_plain, "instances_per_s": len(insts) / t_plain,
                    "cell_updates_per_s": float(np.dot(acc, ncell)) / t_plain,
                    "sample_seconds_per_instance": {str(n): v[0] for n, v in per_size.items()},
                    "sample_per_size": args.ens_plain_sample,
                    "how": "engine.Simulation.run per instance, one at a time; same steps as the batched instance"}
    out["speedup_batched_vs_plain"] = t_plain / t_batch
    out["identical_trajectories"] = True
    if fp64_check:
        out["error_vs_fp64"] = ensemble_fp64_check(insts, args.ens_check_time)
    return out


def ensemble_fp64_check(insts, T, picks=(0, 1)):
    """Two instances (the first of the two smallest sizes present) run by the
    engine -- bit-identical to their ensemble runs -- and by the FP64 oracle
    (oracle/gpu64.py, the checker) to time T: max |dm| per cell and |d<m>|."""
    import torch
    from oracle import gpu64
    from oracle import oracle as O
    from umagnus_b200 import engine
    sizes = sorted({d["N"][0] for d in insts})
    chosen = []
    for n in sizes[: len(picks)]:
        chosen.append(next(i for i, d in enumerate(insts) if d["N"][0] == n))
    res = []
    for i in chosen:
        d = insts[i]
        m0 = random_m(d["N"], d["m_seed"])
        sim = engine.Simulation(d["N"], d["cell"], d["Msat"], d["Aex"], d["alpha"], B_ext=d["B_ext"])
        sim.set_m(m0)
        sim.run(T)
        m32 = sim.get_m().reshape((3,) + sim.shape).double()
        st = sim.state()
        sim.free()
        s64 = gpu64.System64(d["N"], d["cell"], d["Msat"], O.exch_lut(np.full(256, d["Aex"]), dtype=np.float64),
                             np.zeros(d["N"][::-1], np.uint8), d["alpha"], kernel=O.newell_kernel(d["N"], d["cell"]),
                             B_ext=d["B_ext"])
        st64 = gpu64.RK45DP64(s64, m0.astype(np.float64))
        while st64.time < T:
            if st64.time + st64.dt > T:
                st64.dt = T - st64.time
            st64.step()
        dm = float(torch.sqrt(((m32 - st64.m) ** 2).sum(0)).max())
        dav = float(np.abs(m32.reshape(3, -1).mean(1).cpu().numpy() - st64.average_m()).max())
        r = {"instance": i, "N": list(d["N"]), "alpha": d["alpha"], "t": T, "steps_f32": int(st["nsteps"]),
             "steps_f64": st64.nsteps, "max_abs_dm_per_cell": dm, "max_abs_d_avg_m": dav}
        if dm > 1e-3:
            # the reference's float32 arithmetic (the CPU oracle, bit-identical to
            # its kernels) against FP64 on the same instance: at low damping a
            # random state separates float32 from FP64 cell by cell as much
            ref = O.Simulation(d["N"], d["cell"], d["Msat"], d["Aex"], d["alpha"], B_ext=d["B_ext"])
            ref.set_m(m0)
            ref.run(T)
            dr = np.sqrt(((ref.m.astype(np.float64) - st64.m.cpu().numpy()) ** 2).sum(0))
            r["reference_f32_vs_fp64_max_abs_dm_per_cell"] = float(dr.max())
        res.append(r)
    return res


def run_ensemble(args):
    """Batched ensemble vs the plain engine one instance at a time (the
    ensemble workload's own line).  Under torchrun each rank runs its share of
    the instances (partition_instances) and the job's time is the slowest
    rank's."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    out = ensemble_measure(args, rank, world, dist, local_rank, fp64_check=not args.no_fp64_check)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": "RK45DP instances/s, 256-instance thin-film ensemble", "value": out["batched"]["instances_per_s"],
                "unit": "instances/s", "n_gpus": world, "higher_is_better": True,
                "scaling": "strong", "dtype": "f32", "data": "synthetic (seeded instances and m0)",
                "config": {"workload": "256 films n x n x 1, n in {32,48,64,96,128}, 4x4x3 nm, Newell demag + exchange "
                                       "+ Zeeman, RK45DP MaxErr 1e-5, each instance to t = %g s" % args.ens_time,
                           "instances": out["instances"]},
                "ensemble": out}
        print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ adjoint workload
def adjoint_problem(seed=4, m0_kind="easy_axis"):
    """The differentiation workload: 128x128x1 film of 4 nm cubes, per-cell Ms
    U[6e5, 9e5] A/m, Aex 1.3e-11 J/m, Ku1 2e5 J/m^3 along x, alpha 0.02,
    B_ext (5, 5, 0) mT; fixed-step RK4, dt 1e-13 s, 4000 steps, checkpoints
    every 100 steps; loss = mean over the last 1000 steps of m_z averaged over
    a 16x16 probe window (centre of the film) + |<m>(final) - target|^2 with a
    seeded random unit target.  m0 (not fixed by the workload's definition):
    "easy_axis" = uniform along +x, the anisotropy axis, so that the applied
    field drives a damped precession; "random" = i.i.d. random unit vectors,
    whose low-damping dynamics are chaotic (float32 and FP64 runs part after
    a few hundred steps)."""
    rng = np.random.default_rng(seed)
    n = 128
    Ms = rng.uniform(6e5, 9e5, (1, n, n)).astype(np.float32)
    if m0_kind == "random":
        m0 = random_m((n, n, 1), seed + 1)
    else:
        m0 = np.zeros((3, 1, n, n), np.float32)
        m0[0] = 1.0
    t = rng.standard_normal(3)
    t /= np.linalg.norm(t)
    kw = dict(N=(n, n, 1), cell=(4e-9, 4e-9, 4e-9), alpha=0.02, anisU=(1.0, 0.0, 0.0), dt=1e-13, nsteps=4000,
              probe=(56, 56, 16, 16), avg_from=3001, target=tuple(float(x) for x in t))
    theta = dict(Aex=1.3e-11, Ku1=2e5, B_ext=(5e-3, 5e-3, 0.0))
    return kw, Ms, m0, theta


def adjoint_measure(args, fd=True, fp64=True):
    """Forward and backward of the differentiation workload, timed with CUDA
    events (each call returns after its work ends; median of args.adj_reps
    after one warm-up).  fd: central differences of the FP32 forward
    (relative step 1e-4) for Aex, Ku1 and B_ext, and of single Ms cells
    (FP32 resolution limits these).  fp64: the FP64 oracle's reverse pass
    (oracle/adjoint_ref.py, torch float64 on the GPU -- the checker) against
    the GPU gradients, and the oracle's own central differences for Aex, Ku1
    and B_ext against its reverse pass (the 1e-4 agreement at full size).
    Options: --adj-solver (rk4, the workload's stepper, or heun), --adj-steps
    (fewer steps, the probe average over the last quarter), --adj-m0."""
    import torch
    from umagnus_b200.adjoint import AdjointRK4
    kw, Ms, m0, th = adjoint_problem(m0_kind=args.adj_m0)
    if args.adj_steps:
        kw["nsteps"] = args.adj_steps
        kw["avg_from"] = args.adj_steps - args.adj_steps // 4 + 1
    nsteps = kw["nsteps"]
    solver = 2 if args.adj_solver == "heun" else 4
    sim = AdjointRK4(K=min(100, nsteps), solver=solver, **kw)
    sname = "Heun" if solver == 2 else "RK4"
    fw, bw = [], []
    for it in range(1 + args.adj_reps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        loss = sim.forward(m0, Ms, th["Aex"], th["Ku1"], th["B_ext"])
        e1.record()
        g = sim.backward()
        e2.record()
        torch.cuda.synchronize()
        if it >= 1:
            fw.append(e0.elapsed_time(e1) / 1e3)
            bw.append(e1.elapsed_time(e2) / 1e3)
    f, b = float(np.median(fw)), float(np.median(bw))
    N = 128 * 128
    gMs = g["Ms"].cpu().numpy()
    cells = np.random.default_rng(7).choice(N, 64, replace=False)
    out = {"workload": "128x128x1 film, 4 nm cells, per-cell Ms U[6e5,9e5], Aex 1.3e-11, Ku1 2e5 along x, "
                       f"alpha 0.02, B_ext (5,5,0) mT, Newell demag, fixed-step {sname} dt 1e-13 s x {nsteps}, "
                       f"checkpoints every {min(100, nsteps)} steps",
           "m0": "uniform along +x" if args.adj_m0 == "easy_axis" else "random unit vectors",
           "forward_s": f, "backward_s": b, "backward_over_forward": b / f, "target": "<= 3",
           "forward_cell_updates_per_s": nsteps * N / f, "loss": loss,
           "grad": {"Aex": g["Aex"], "Ku1": g["Ku1"], "B_ext": g["B_ext"],
                    "Ms_norm": float(np.linalg.norm(gMs.astype(np.float64)))}}

    def rel(a, b_):
        a, b_ = np.asarray(a, np.float64), np.asarray(b_, np.float64)
        return float(np.linalg.norm(a - b_) / np.linalg.norm(b_))

    d = 1e-4
    Bn = float(np.linalg.norm(th["B_ext"]))

    def central(L, grad_key=None):
        r = {"Aex": (L(A=th["Aex"] * (1 + d)) - L(A=th["Aex"] * (1 - d))) / (2 * d * th["Aex"]),
             "Ku1": (L(K=th["Ku1"] * (1 + d)) - L(K=th["Ku1"] * (1 - d))) / (2 * d * th["Ku1"])}
        fdB = []
        for c in range(3):
            bp, bm = list(th["B_ext"]), list(th["B_ext"])
            bp[c] += d * Bn
            bm[c] -= d * Bn
            fdB.append((L(B=bp) - L(B=bm)) / (2 * d * Bn))
        r["B_ext"] = fdB
        return r

    if fd:
        def L32(Ms_=Ms, A=th["Aex"], K=th["Ku1"], B=th["B_ext"]):
            return sim.forward(m0, Ms_, A, K, B)
        c32 = central(L32)
        errs = []
        for c in cells[:8]:
            mp, mm = Ms.copy().ravel(), Ms.copy().ravel()
            hM = d * float(Ms.ravel()[c])
            mp[c] += hM
            mm[c] -= hM
            v = (L32(Ms_=mp.reshape(Ms.shape)) - L32(Ms_=mm.reshape(Ms.shape))) / (2 * hM)
            errs.append(abs(v - gMs.ravel()[c]) / max(abs(v), 1e-300))
        out["fd_fp32"] = {"rel_step": d, "Aex": [c32["Aex"], g["Aex"]], "Ku1": [c32["Ku1"], g["Ku1"]],
                          "B_ext": [c32["B_ext"], g["B_ext"]],
                          "rel_err_Aex": abs(c32["Aex"] - g["Aex"]) / abs(c32["Aex"]),
                          "rel_err_Ku1": abs(c32["Ku1"] - g["Ku1"]) / abs(c32["Ku1"]),
                          "rel_err_B_ext": rel(g["B_ext"], c32["B_ext"]),
                          "Ms_8_cells_rel_err_median": float(np.median(errs)),
                          "note": "FP32 central differences resolve the loss to ~1e-7: single-cell Ms steps "
                                  "move it below that (checked in FP64 below)"}
    if fp64:
        from oracle import adjoint_ref as R
        t0 = time.perf_counter()
        prob = R.Problem(solver=solver, backend="torch", device="cuda", **kw)
        th64 = R.params(Ms.astype(np.float64), th["Aex"], th["Ku1"], th["B_ext"])
        loss64, g64 = prob.backward(m0.astype(np.float64).reshape(3, 1, 128, 128), th64)
        per_cell = np.abs(gMs.ravel()[cells] - g64["Ms"].ravel()[cells]) / np.abs(g64["Ms"].ravel()[cells])
        out["fp64_reverse"] = {"loss_fp64": loss64, "loss_rel_err": abs(loss - loss64) / abs(loss64),
                               "rel_err": {"Ms": rel(gMs, g64["Ms"]), "Aex": rel(g["Aex"], g64["A"]),
                                           "Ku1": rel(g["Ku1"], g64["K1"]), "B_ext": rel(g["B_ext"], g64["B"]),
                                           "m0": rel(g["m0"].cpu().numpy(), g64["m0"])},
                               "Ms_64_cells_max_rel_err": float(per_cell.max()),
                               "seconds": time.perf_counter() - t0}
        if fd:
            t0 = time.perf_counter()

            def L64(A=th["Aex"], K=th["Ku1"], B=th["B_ext"]):
                return prob.forward(m0.astype(np.float64).reshape(3, 1, 128, 128),
                                    R.params(Ms.astype(np.float64), A, K, B))
            c64 = central(L64)
            out["fd_fp64"] = {"rel_step": d,
                              "rel_err_reverse_vs_fd": {"Aex": abs(c64["Aex"] - g64["A"]) / abs(c64["Aex"]),
                                                        "Ku1": abs(c64["Ku1"] - g64["K1"]) / abs(c64["Ku1"]),
                                                        "B_ext": rel(g64["B"], c64["B_ext"])},
                              "rel_err_gpu_vs_fd": {"Aex": abs(c64["Aex"] - g["Aex"]) / abs(c64["Aex"]),
                                                    "Ku1": abs(c64["Ku1"] - g["Ku1"]) / abs(c64["Ku1"]),
                                                    "B_ext": rel(g["B_ext"], c64["B_ext"])},
                              "target": "<= 1e-4", "seconds": time.perf_counter() - t0}
    sim.free()
    return out


def run_adjoint(args):
    """The differentiation workload's own line: backward/forward time and the
    gradient checks (adjoint_measure; --adj-fd, --adj-fp64 select them)."""
    out = adjoint_measure(args, fd=args.adj_fd, fp64=args.adj_fp64)
    line = {"metric": "adjoint backward/forward time, 128x128x1 film", "value": out["backward_over_forward"],
            "unit": "backward/forward", "n_gpus": 1, "higher_is_better": False, "dtype": "f32",
            "data": "synthetic (seeded Ms map, m0 and target)", "config": {"workload": out["workload"]},
            "adjoint": out}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ thin-film comparison workload
def run_fieldevals(args):
    """A short run of the multilayer's field + torque evaluations and of the
    three demag passes one by one (--steps evaluations after --warmup): the
    target for kernel profilers, whose launch list holds only these kernels.
    Prints the evaluation and pass times (CUDA events)."""
    import torch
    from umagnus_b200 import engine
    torch.cuda.set_device(0)
    cfg = CONFIG
    N = cfg["N"]
    sim = engine.Simulation(N, cfg["cell"], cfg["Ms"], cfg["Aex"], cfg["alpha"], Dind=cfg["Dind"], Ku1=cfg["Ku1"],
                            anisU=cfg["anisU"], B_ext=cfg["B_ext"], device=0)
    sim.set_m(random_m(N, cfg["seed"]))
    stream = torch.cuda.Stream()
    sim.set_stream(stream)
    sim.torque_evals(max(args.warmup, 1))
    stream.synchronize()
    E = max(args.steps, 1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.torque_evals(E)
    e1.record(stream)
    e1.synchronize()
    ms_pass = time_passes(N, cfg["cell"], cfg["Ms"], stream, reps=E)
    print(json.dumps({"workload": "fieldevals", "N": list(N), "evals": E, "us_per_eval": e0.elapsed_time(e1) / E * 1e3,
                      "us_per_pass": {k: v * 1e3 for k, v in ms_pass.items()}}))
    return 0


def run_film(args):
    """The plain thin film (64x64x1 cells of 4x4x3 nm, Ms 8e5 A/m, Aex
    1.3e-11 J/m, alpha 0.1, B_ext (0, 0, 10 mT), no anisotropy, m0 random
    unit vectors from a seed, Newell demag, RK45DP MaxErr 1e-5 to 1 ns) on the
    GPU engine, beside the reference's float32 kernels on the host cores
    (oracle/ref_arm.py: the reference's OpenCL C kernels compiled for the
    host, scipy FFT, the RK45DP controller restated) and the FP64 oracle on the
    GPU: the average-m time series compared on a common time grid, the final
    m per cell, step counts and wall times."""
    import torch
    from oracle import gpu64
    from oracle import oracle as O
    from oracle.ref_arm import RefRK45
    from umagnus_b200 import engine
    N, cell, T = (64, 64, 1), (4e-9, 4e-9, 3e-9), args.film_time
    Ms, Aex, alpha, B = 8e5, 1.3e-11, 0.1, (0.0, 0.0, 0.01)
    m0 = random_m(N, 1)
    # GPU engine: wall time of the plain run, then the series step by step
    sim = engine.Simulation(N, cell, Ms, Aex, alpha, B_ext=B)
    sim.set_m(m0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.run(T)
    torch.cuda.synchronize()
    t_gpu = time.perf_counter() - t0
    st_gpu = sim.state()
    m_gpu = sim.get_m().cpu().numpy().reshape(m0.shape)
    sim.free()
    sim = engine.Simulation(N, cell, Ms, Aex, alpha, B_ext=B)
    sim.set_m(m0)
    ser_gpu = [(0.0, np.array(sim.average_m()))]
    while sim.state()["time"] < T:
        before = sim.state()["nsteps"]
        sim.run(T - sim.state()["time"], chunk=1, max_steps=1)
        if sim.state()["nsteps"] > before:
            ser_gpu.append((sim.state()["time"], np.array(sim.average_m())))
    sim.free()
    # reference kernels on the host
    orc = O.Simulation(N, cell, Ms, Aex, alpha, B_ext=B)
    ref = RefRK45(N, cell, Ms, Aex, alpha, 0.0, 0.0, (0.0, 0.0, 1.0), B, Kf=orc.Kf)
    orc.set_m(m0)
    ref.set_m(orc.m)
    ref.alarm = T
    ser_ref = [(0.0, ref.m.reshape(3, -1).mean(1).astype(np.float64))]
    t0 = time.perf_counter()
    while ref.time < T:
        if ref.step():
            ser_ref.append((ref.time, ref.m.reshape(3, -1).mean(1).astype(np.float64)))
    t_ref = time.perf_counter() - t0
    # FP64 oracle on the GPU
    sys64 = gpu64.System64(N, cell, Ms, O.exch_lut(np.full(256, Aex), dtype=np.float64), np.zeros(N[::-1], np.uint8),
                           alpha, kernel=O.newell_kernel(N, cell), B_ext=B)
    st64 = gpu64.RK45DP64(sys64, orc.m.astype(np.float64))
    ser64 = [(0.0, st64.average_m())]
    while st64.time < T:
        st64.dt = min(st64.dt, T - st64.time) if st64.time + st64.dt > T else st64.dt
        if st64.step():
            ser64.append((st64.time, st64.average_m()))
    grid = np.linspace(0.0, T, 201)

    def interp(ser):
        t = np.array([x[0] for x in ser])
        a = np.array([x[1] for x in ser])
        return np.stack([np.interp(grid, t, a[:, c]) for c in range(3)], axis=1)

    g, r, f = interp(ser_gpu), interp(ser_ref), interp(ser64)
    dm_ref = np.abs(m_gpu - ref.m).max()
    dm_64 = float(np.abs(m_gpu - st64.m.cpu().numpy()).max())
    line = {"metric": "thin film 64x64x1 to 1 ns: GPU engine vs reference float32 kernels on the host",
            "value": float(np.abs(g - r).max()), "unit": "max |d<m>| over the run",
            "higher_is_better": False, "dtype": "f32", "n_gpus": 1, "data": "synthetic (seeded random m0)",
            "config": {"workload": "64x64x1 cells of 4x4x3 nm, Ms 8e5, Aex 1.3e-11, alpha 0.1, B_ext (0,0,10 mT), "
                                   f"Newell demag, RK45DP MaxErr 1e-5, t = 0..{T:g} s"},
            "avg_m_max_abs_diff": {"gpu_vs_reference_f32": float(np.abs(g - r).max()),
                                   "gpu_vs_fp64": float(np.abs(g - f).max()),
                                   "reference_f32_vs_fp64": float(np.abs(r - f).max())},
            "final_avg_m": {"gpu": g[-1].tolist(), "reference_f32": r[-1].tolist(), "fp64": f[-1].tolist()},
            "final_m_max_abs_diff": {"gpu_vs_reference_f32": float(dm_ref), "gpu_vs_fp64": dm_64},
            "accepted_steps": {"gpu": int(st_gpu["nsteps"]), "reference_f32": ref.nsteps, "fp64": st64.nsteps},
            "rejected_steps": {"gpu": int(st_gpu["nundone"]), "reference_f32": ref.nundone, "fp64": st64.nundone},
            "wall_s": {"gpu": t_gpu, "reference_f32_cpu": t_ref, "reference_threads": ref.threads},
            "speedup_vs_reference_cpu": t_ref / t_gpu}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ precision workload
def voronoi_grains(N, ngrain, seed):
    """Columnar Voronoi grains: ngrain seed points uniform in the film plane
    (seeded), each cell (and the column above it) in the grain of its nearest
    seed; grain index = region id."""
    rng = np.random.default_rng(seed)
    Nx, Ny, Nz = N
    pts = rng.uniform(0, 1, size=(ngrain, 2)) * np.array([Nx, Ny])
    x = np.arange(Nx) + 0.5
    y = np.arange(Ny) + 0.5
    best = np.full((Ny, Nx), np.inf)
    grain = np.zeros((Ny, Nx), np.uint8)
    for g, (px, py) in enumerate(pts):
        d = (x[None, :] - px) ** 2 + (y[:, None] - py) ** 2
        closer = d < best
        best[closer] = d[closer]
        grain[closer] = g
    return np.broadcast_to(grain, (Nz, Ny, Nx)).copy()


def precision_problem(N=(512, 512, 32), seed=3):
    """The precision workload: 2 nm cubes, 64 columnar Voronoi grains (region
    ids 0..63), each grain of class 0 or 1 (seeded) with Ms 6e5 / 9e5 A/m and
    Aex 1.0e-11 / 1.5e-11 J/m, Ku1 2e5 J/m^3 along a random axis per grain
    (seeded), alpha 0.05, no applied field, m0 random unit vectors (seeded)."""
    rng = np.random.default_rng(seed)
    regions = voronoi_grains(N, 64, seed)
    cls = rng.integers(0, 2, size=64)
    ms_r = np.where(cls == 0, 6e5, 9e5)
    aex_r = np.zeros(256)
    aex_r[:64] = np.where(cls == 0, 1.0e-11, 1.5e-11)
    axes = rng.standard_normal((64, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    Ms = ms_r[regions].astype(np.float32)
    u = np.stack([axes[regions][..., c] for c in range(3)]).astype(np.float32)
    m0 = random_m(N, seed + 1)
    return dict(N=N, cell=(2e-9, 2e-9, 2e-9), regions=regions, Ms=Ms, aex_r=aex_r, Ku1=2e5, u=u, alpha=0.05, m0=m0)


def run_precision(args):
    """Float32 engine (FP64 Newell tensor, compensated sums, FP64 time) against
    the FP64 instantiation of the oracle on the GPU (oracle/gpu64.py, the
    uMagNUS64 semantics) from the same m0: the effective field and energy
    density of the same m (at m0 and at the final float32 state), then
    --prec-steps RK45DP step attempts on both, comparing average m and the
    accepted dt sequence step by step."""
    import torch
    from oracle import gpu64
    from oracle import oracle as O
    from umagnus_b200 import engine
    from umagnus_b200 import opencl as cl
    N = tuple(int(v) for v in args.prec_size.split("x"))
    pb = precision_problem(N)
    t_start = time.perf_counter()
    sim = engine.Simulation(N, pb["cell"], Msat=pb["Ms"], Aex=pb["aex_r"], alpha=pb["alpha"], Ku1=pb["Ku1"],
                            anisU=pb["u"], regions=pb["regions"])
    sim.set_m(pb["m0"])
    d = cl.NewNewellDemag(N, (0, 0, 0), pb["cell"])
    K = d.kernel()
    d.Free()
    sys64 = gpu64.System64(N, pb["cell"], pb["Ms"].astype(np.float64), O.exch_lut(pb["aex_r"], dtype=np.float64),
                           pb["regions"], pb["alpha"], kernel=K, Ku1=pb["Ku1"], anisU=pb["u"].astype(np.float64))
    del K

    def field_errors(label):
        m32 = sim.get_m().reshape((3,) + sim.shape)
        _, B32 = sim.torque(beff=True)
        B32 = B32.reshape((3,) + sim.shape).double()
        e32 = sim.energy_density().double()
        m = m32.double()
        B64 = sys64.beff(m)
        e64 = sys64.energy_density(m)
        dB = torch.sqrt(((B32 - B64) ** 2).sum(0))
        nB = torch.sqrt((B64 ** 2).sum(0))
        de = (e32 - e64).abs()
        return {label: {"B_eff": {"max_abs_T": float(dB.max()), "rms_abs_T": float(torch.sqrt((dB ** 2).mean())),
                                  "max_rel_to_max": float(dB.max() / nB.max()),
                                  "rms_rel_to_rms": float(torch.sqrt((dB ** 2).mean() / (nB ** 2).mean()))},
                        "energy_density": {"max_abs_J_m3": float(de.max()),
                                           "rms_abs_J_m3": float(torch.sqrt((de ** 2).mean())),
                                           "max_rel_to_max": float(de.max() / e64.abs().max()),
                                           "rms_rel_to_rms": float(torch.sqrt((de ** 2).mean() / (e64 ** 2).mean()))},
                        "total_energy_rel": float(abs(e32.sum() - e64.sum()) / abs(e64.sum()))}}

    out = field_errors("at_m0")
    st64 = gpu64.RK45DP64(sys64, sim.get_m().reshape((3,) + sim.shape).double().cpu().numpy())
    rec32, rec64 = [], []
    prev = sim.state()
    for i in range(args.prec_steps):
        sim.steps(1)
        s = sim.state()
        acc = s["nsteps"] > prev["nsteps"]
        rec32.append((acc, s["time"] - prev["time"], s["dt"], sim.average_m()))
        prev = s
        t0 = st64.time
        a64 = st64.step()
        rec64.append((a64, st64.time - t0, st64.dt, st64.average_m()))
    same = 0
    while same < len(rec32) and rec32[same][0] == rec64[same][0]:
        same += 1
    dts32 = np.array([r[1] for r in rec32[:same] if r[0]])
    dts64 = np.array([r[1] for r in rec64[:same] if r[0]])
    rel_dt = np.abs(dts32 - dts64) / dts64
    am32 = np.array([r[3] for r in rec32[:same]])
    am64 = np.array([r[3] for r in rec64[:same]])
    dam = np.linalg.norm(am32 - am64, axis=1)
    out.update(field_errors("at_final_state"))
    mf32 = sim.get_m().reshape((3,) + sim.shape).double()
    dm = torch.sqrt(((mf32 - st64.m) ** 2).sum(0))
    line = {"metric": "float32 engine error against the FP64 oracle (precision workload)",
            "value": float(rel_dt.max()) if rel_dt.size else None, "unit": "max relative error of accepted dt",
            "higher_is_better": False, "dtype": "f32", "n_gpus": 1,
            "data": "synthetic (seeded Voronoi grains, axes, m0)",
            "config": {"workload": f"{N[0]}x{N[1]}x{N[2]} cells of 2 nm, 64 Voronoi grains (2 classes: Ms 6e5/9e5, "
                                   "Aex 1.0e-11/1.5e-11), Ku1 2e5 along a random axis per grain, alpha 0.05, "
                                   "Newell demag, RK45DP MaxErr 1e-5",
                       "step_attempts": args.prec_steps, "oracle": "oracle/gpu64.py (FP64, torch + cuFFT)"},
            "fields": out,
            "trajectory": {"attempts_with_identical_accept_decisions": same,
                           "accepted_f32": int(sum(r[0] for r in rec32)), "accepted_f64": int(sum(r[0] for r in rec64)),
                           "time_f32": prev["time"], "time_f64": st64.time,
                           "dt_rel_err": {"max": float(rel_dt.max()) if rel_dt.size else None,
                                          "rms": float(np.sqrt((rel_dt ** 2).mean())) if rel_dt.size else None},
                           "avg_m_abs_err": {"max": float(dam.max()) if dam.size else None,
                                             "rms": float(np.sqrt((dam ** 2).mean())) if dam.size else None,
                                             "final": float(dam[-1]) if dam.size else None},
                           "final_m_per_cell_err": {"max": float(dm.max()), "rms": float(torch.sqrt((dm ** 2).mean()))},
                           "avg_m_abs_err_at_attempt": {str(k): float(dam[k - 1]) for k in (10, 100, 250, 500, 1000, 1500, 2000)
                                                        if k <= dam.size},
                           "dt_rel_err_at_accepted": {str(k): float(rel_dt[k - 1]) for k in (10, 100, 250, 500, 1000, 1500, 2000)
                                                      if k <= rel_dt.size}},
            "seconds": time.perf_counter() - t_start}
    print(json.dumps(line), flush=True)
    return 0


def spawn_ranks(n):
    """--gpus N without a launcher: start N ranks, one process per GPU, with
    torch.distributed.run on 127.0.0.1 and the same arguments (rank 0 prints
    the line); fails if fewer than N GPUs are visible."""
    import socket
    import subprocess

    import torch
    have = torch.cuda.device_count()
    if have < n:
        print(json.dumps({"error": f"--gpus {n} asked for {n} GPUs, {have} visible"}), flush=True)
        return 2
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="multilayer: default launch shapes, no search")
    ap.add_argument("--ref-budget", type=float, default=90.0, help="seconds of timed CPU steps (reference arm)")
    ap.add_argument("--workload", default="multilayer",
                    choices=["multilayer", "ensemble", "adjoint", "precision", "film", "fieldevals"])
    ap.add_argument("--adj-fp64", action="store_true", help="adjoint: compare with the FP64 oracle (minutes of CPU)")
    ap.add_argument("--adj-fd", action="store_true", help="adjoint: central differences of the FP32 forward")
    ap.add_argument("--adj-steps", type=int, default=0, help="adjoint: steps instead of 4000")
    ap.add_argument("--prec-steps", type=int, default=2000, help="precision: RK45DP step attempts")
    ap.add_argument("--film-time", type=float, default=1e-9, help="film: simulated time (s)")
    ap.add_argument("--prec-size", default="512x512x32", help="precision: mesh NxxNyxNz")
    ap.add_argument("--adj-m0", default="easy_axis", choices=["easy_axis", "random"], help="adjoint: initial m")
    ap.add_argument("--adj-solver", default="rk4", choices=["rk4", "heun"], help="adjoint: fixed-step stepper")
    ap.add_argument("--ens-time", type=float, default=2e-9, help="ensemble: simulated time per instance (s)")
    ap.add_argument("--ens-plain-sample", type=int, default=2, help="ensemble: plain-form instances timed per size")
    ap.add_argument("--ens-check-time", type=float, default=2e-11, help="ensemble: FP64 check horizon (s)")
    ap.add_argument("--adj-reps", type=int, default=2, help="adjoint: timed forward/backward repetitions")
    ap.add_argument("--no-ensemble", action="store_true", help="multilayer line: skip the ensemble sub-object")
    ap.add_argument("--no-adjoint", action="store_true", help="multilayer line: skip the adjoint sub-object")
    ap.add_argument("--no-fp64-check", action="store_true", help="skip the FP64 oracle checks")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    if args.workload == "ensemble":
        return run_ensemble(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "film":
        return run_film(args)
    if args.workload == "fieldevals":
        return run_fieldevals(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        r = make_ref(CONFIG)
        for _ in range(min(max(args.warmup, 1), 2)):  # bounded warm-up: a CPU step takes seconds
            r.step()
        t, n, acc = time_ref(r, args.steps, args.ref_budget)
        ncell = r.n
        value = acc * ncell / t
        sample = (f"{n} of the {args.steps} requested RK45DP steps ({acc} accepted, {t:.1f} s budget-bounded) of "
                  f"the full workload: reference OpenCL C kernels compiled for the host on {r.threads} threads, "
                  "scipy.fft (multi-threaded) standing in for the reference's VkFFT")
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": n,
                "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": t / n * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded random m)", "impl": "reference",
                "config": {"workload": "multilayer 256x256x16 cells 2x2x1 nm, DMI + uniaxial + Zeeman + Newell "
                                       "demag, RK45DP adaptive, MaxErr 1e-5", "cells": ncell},
                "cpu_baseline": {"kind": "reference", "cores": r.threads, "sample": sample, "value": value,
                                 "unit": UNIT},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_ours(args, rank, world, local_rank)
    dist_mod = None
    if world > 1:
        import torch.distributed as dist_mod
    # the ensemble (sharded over the ranks, no collective during the run) and,
    # at N = 1, the differentiation workload: the batched-against-plain and
    # backward-over-forward figures, measured in the same run (outside the
    # multilayer's timed region)
    if not args.no_ensemble:
        ens = ensemble_measure(args, rank, world, dist_mod, local_rank, plain=(world == 1),
                               fp64_check=not args.no_fp64_check)
        if rank == 0:
            res["ensemble"] = ens
    if rank == 0:
        if world == 1 and not args.no_adjoint:
            res["adjoint"] = adjoint_measure(args, fd=True, fp64=not args.no_fp64_check)
        if world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(CONFIG)
        print(json.dumps(res), flush=True)
    if world > 1:
        dist_mod.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
