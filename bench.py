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

--impl reference times the reference's CPU implementation of the path: the
reference's own OpenCL C kernels compiled for the host (oracle/_ref), with
the FFT and the engine loop restated (oracle/), on one host thread.
"""
import argparse
import json
import os
import subprocess
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


def random_m(N, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((3, N[2], N[1], N[0]))
    v /= np.sqrt((v * v).sum(axis=0))
    return v.astype(np.float32)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU baseline
def cpu_baseline(config):
    """Time one field + torque evaluation and one RK45DP stage-sum set of the
    full workload on one host thread (reference kernels via oracle/_ref when
    built, else the oracle port); the step time is 6 evaluations + 7 stage
    sums + the error combination."""
    from oracle import clref
    from oracle import oracle as O
    N, cell = config["N"], config["cell"]
    t0 = time.perf_counter()
    K = O.newell_kernel(N, cell)
    Kf, _ = O.kernel_spectrum(K)
    del K
    t_setup = time.perf_counter() - t0
    m = random_m(N, config["seed"])
    n = m[0].size
    P = O.pad_size(N)
    kind = "reference" if clref.available() else "port"
    alut = O.exch_lut(np.full(256, config["Aex"], np.float32))
    dlut = O.exch_lut(np.full(256, config["Dind"], np.float32))
    regions = np.zeros(m.shape[1:], np.uint8)
    lut = np.zeros((3, 256), np.float32)
    lut[:] = np.asarray(config["B_ext"], np.float32)[:, None]
    t1 = time.perf_counter()
    B = O.demag_field(Kf, P, m, config["Ms"], dtype=np.float32)
    if kind == "reference":
        c = [float(np.float32(x)) for x in cell]
        clref.call("adddmi", np.float32, B[0], B[1], B[2], m[0], m[1], m[2], None, config["Ms"], alut, dlut, regions,
                   c[0], c[1], c[2], N[0], N[1], N[2], 0, 0)
        clref.call("adduniaxialanisotropy2", np.float32, B[0], B[1], B[2], m[0], m[1], m[2], None, config["Ms"],
                   None, config["Ku1"], None, 0.0, None, 0.0, None, 0.0, None, 1.0, n)
        clref.call("regionaddv", np.float32, B[0], B[1], B[2], lut[0], lut[1], lut[2], regions, n)
        clref.call("lltorque2", np.float32, B[0], B[1], B[2], m[0], m[1], m[2], B[0], B[1], B[2], None,
                   config["alpha"], n)
    else:
        O.add_dmi(B, m, alut, dlut, regions, cell, config["Ms"])
        O.add_uniaxial(B, m, config["Ms"], config["Ku1"], 0.0, config["anisU"])
        O.region_addv(B, lut, regions)
        B = O.lltorque(m, B, config["alpha"])
    t_eval = time.perf_counter() - t1
    # stage sums: 3+4+5+6+7+7 source vectors over 6 stages + error (6 sources)
    t2 = time.perf_counter()
    ks = [B.copy() for _ in range(7)]
    for nsrc in (2, 3, 4, 5, 6, 6):
        srcs = [m] + ks[: nsrc - 1]
        out = np.stack([O.madd([s[cc].ravel() for s in srcs], [1.0] + [1e-3] * (nsrc - 1)) for cc in range(3)])
        mm = out.reshape(m.shape)
        O.normalize(mm)
    O.max_vec_norm(ks[0])
    t_stage = time.perf_counter() - t2
    t_step = 6 * t_eval + t_stage
    return {"value": n / t_step, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": (f"one field+torque evaluation ({t_eval:.1f} s) and one set of RK45DP stage sums "
                       f"({t_stage:.1f} s) of the full 256x256x16 workload on 1 host thread; step = 6 evals + "
                       f"stage sums; kernel setup {t_setup:.1f} s excluded")}


# ------------------------------------------------------------------ GPU arm
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
    stream = torch.cuda.Stream()
    sim.set_stream(stream)
    m0 = random_m(N, cfg["seed"] + rank)
    sim.set_m(m0)
    graph_steps = 16
    sim.use_graph(True, graph_steps)
    # warm-up (also builds the CUDA graph)
    sim.steps(max(args.warmup, 3))
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
    # end-to-end through the public API with host buffers
    host_m = torch.from_numpy(m0).pin_memory()
    host_out = torch.empty_like(host_m).pin_memory()
    dev_m = torch.empty_like(host_m, device="cuda")
    torch.cuda.synchronize()
    t_e0 = time.perf_counter()
    dev_m.copy_(host_m, non_blocking=True)
    sim.set_m(dev_m)
    chunks = max(1, args.steps // graph_steps)
    s_before = sim.state()
    for _ in range(chunks):
        sim.steps(graph_steps)
        s_now = sim.state()  # D2H of the solver state after every chunk
    out = sim.get_m()
    host_out.copy_(out)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t_e0
    acc_e2e = s_now["nsteps"] - s_before["nsteps"]
    steps_e2e = chunks * graph_steps
    bytes_state = 88
    times = torch.tensor([ms, ms_eval, t_e2e], dtype=torch.float64, device="cuda")
    accs = torch.tensor([acc, acc_e2e], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(times, op=dist.ReduceOp.MAX)
        dist.all_reduce(accs, op=dist.ReduceOp.SUM)
    ms_max, ms_eval_max, t_e2e_max = times.tolist()
    acc_tot, acc_e2e_tot = accs.tolist()
    result = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        b_eval = alg_bytes_per_eval(N)
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
                       "graph_steps": graph_steps},
            "roofline": {"bound": "hbm", "kernel": "field+torque evaluation (demag passes A,B,C + local/torque)",
                         "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "alg_bytes_per_launch": b_eval,
                         "ms_per_eval": ms_eval_max},
            "e2e": {"value": acc_e2e_tot * ncell / t_e2e_max, "unit": UNIT,
                    "h2d_bytes_per_step": (12 * ncell) / steps_e2e,
                    "d2h_bytes_per_step": (12 * ncell + bytes_state * chunks) / steps_e2e,
                    "how": "pinned host m -> device, set_m, steps in graph chunks of 16 with a solver-state "
                           "read-back per chunk, final m -> pinned host; wall clock"},
            "gpu_launches": sim.launches_per_step() * args.steps,
            "clocks": clk.summary(),
        }
    sim.free()
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        res = cpu_baseline(CONFIG)
        line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": CONFIG["N"][0] * CONFIG["N"][1] * CONFIG["N"][2] /
                res["value"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded random m)", "impl": "reference",
                "config": {"workload": "multilayer 256x256x16 cells 2x2x1 nm, DMI + uniaxial + Zeeman + Newell "
                                       "demag, RK45DP"},
                "cpu_baseline": {"kind": res["kind"], "cores": res["cores"], "sample": res["sample"],
                                 "value": res["value"], "unit": UNIT},
                "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_ours(args, rank, world, local_rank)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(CONFIG)
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
