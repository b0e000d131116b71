"""The benchmark's multi-GPU bookkeeping (replicas, one process per GPU) on
CPU ranks over gloo: timings reduce to the slowest rank, step counts to
their sum, so the whole-job throughput is all ranks' cell-updates over the
slowest rank's time; every rank takes the same collective steps."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        times = torch.tensor([10.0 + rank, 2.0 - 0.5 * rank, 3.0 * (rank + 1)], dtype=torch.float64)
        counts = torch.tensor([100.0 + rank, 7.0], dtype=torch.float64)
        t, c = bench.combine_ranks(times, counts, dist)
        dist.barrier()
        out.put((rank, t, c))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_combine_ranks_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, c in res:
        assert t == [10.0 + world - 1, 2.0, 3.0 * world]
        assert c == [100.0 * world + sum(range(world)), 7.0 * world]


def test_combine_ranks_single_process():
    import bench
    t, c = bench.combine_ranks(torch.tensor([1.5, 2.5]), torch.tensor([4.0]), None)
    assert t == [1.5, 2.5] and c == [4.0]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_instances(world):
    """Every instance on exactly one rank, loads within one largest mesh."""
    import bench
    insts = bench.ensemble_instances()
    parts = bench.partition_instances(insts, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(insts)))
    loads = [sum(insts[i]["N"][0] * insts[i]["N"][1] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(d["N"][0] * d["N"][1] for d in insts)


class _StubEnsemble:
    """Stands in for engine.Ensemble on CPU ranks: an instance of n x n cells
    'takes' n steps, and run() records its simulated time."""

    def __init__(self, insts):
        self.insts = insts
        self.set = set()

    def set_m(self, i, m):
        assert m.shape == (3, 1) + tuple(self.insts[i]["N"][:2][::-1])
        self.set.add(i)

    def run(self, T, chunk=8):
        assert self.set == set(range(len(self.insts)))
        self.T = T

    def state(self, i):
        return {"nsteps": self.insts[i]["N"][0], "time": self.T}

    def free(self):
        pass


def _ens_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        insts = bench.ensemble_instances(count=24, seed=9)
        r = bench.ensemble_shard(insts, 1e-12, rank, world, dist, _StubEnsemble, device="cpu")
        t, cells, n, alg, mine, states = r
        out.put((rank, n, cells, alg, [d["m_seed"] for d in mine]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ensemble_shards_over_gloo_ranks(world):
    """The sharded ensemble's rank logic with a stub engine: every instance
    runs on exactly one rank, and every rank reports the job's totals."""
    import bench
    insts = bench.ensemble_instances(count=24, seed=9)
    want_cells = float(sum(d["N"][0] * d["N"][1] * d["N"][0] for d in insts))
    want_alg = float(sum(d["N"][0] * bench.alg_bytes_per_step(d["N"]) for d in insts))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ens_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds = sorted(s for r in res for s in r[4])
    assert seeds == sorted(d["m_seed"] for d in insts)
    for rank, n, cells, alg, _ in res:
        assert n == len(insts) and cells == want_cells and alg == pytest.approx(want_alg, rel=1e-12)


def test_gpus_beyond_visible_fail_loudly():
    """--gpus N with fewer GPUs visible exits with an error line, not a
    one-GPU run reported as N."""
    import json
    import subprocess
    import sys
    from tests.conftest import ROOT
    if torch.cuda.is_available() and torch.cuda.device_count() >= 64:
        pytest.skip("64 GPUs visible")
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "64", "--steps", "1"],
                       capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 2
    assert "64 GPUs" in json.loads(r.stdout.strip().splitlines()[-1])["error"]
