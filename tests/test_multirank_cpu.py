"""Multi-process paths of bench.py on the CPU (gloo, world size 2): the
replicas' host-side barrier and max-over-ranks reduction, the sharding of
the parameter sweep's independent networks over ranks and the reduction of
its per-rank figures, and a full torchrun launch of the reference arm in
which rank 0 alone prints the JSON line and every rank exits 0."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    w, r, _ = bench.dist_setup(None)
    bench.barrier(w)
    m = bench.reduce_max(float(10 * (r + 1)), w)
    with open(os.path.join(out_dir, "rank%d.txt" % r), "w") as f:
        f.write("%d %d %.1f" % (w, r, m))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_gloo_barrier_and_max_over_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        w, rr, m = open(tmp_path / ("rank%d.txt" % r)).read().split()
        assert int(w) == 2 and int(rr) == r and float(m) == 20.0


def test_sweep_sharding_by_size():
    sys.path.insert(0, ROOT)
    import bench
    from tests import sweep
    grid = sweep.sweep_grid(256, 1000, 50000, 100, 500, seed=2024)
    sizes = [p["n"] for p in grid]
    for world in (1, 2, 4, 8):
        shards = bench.shard_networks(sizes, world)
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(len(sizes)))          # every network once
        loads = [sum(sizes[i] for i in sh) for sh in shards]
        # greedy largest-first: no rank carries more than the mean plus the
        # largest network
        assert max(loads) <= sum(sizes) / world + max(sizes)
        assert bench.shard_networks(sizes, world) == shards   # deterministic


def _sweep_worker(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    w, r, _ = bench.dist_setup(None)
    local = {"device_ms": 100.0 + 50.0 * r, "evals": 600.0 * (r + 1), "spikes": 3.0 * (r + 1),
             "neuron_steps": 100.0 * (r + 1), "neurons": 10.0 * (r + 1)}
    tot = bench.sweep_phase_totals(local, w)
    with open(os.path.join(out_dir, "sweep%d.json" % r), "w") as f:
        json.dump(tot, f)
    import torch.distributed as dist
    dist.destroy_process_group()


def test_sweep_phase_totals_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_sweep_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        tot = json.load(open(tmp_path / ("sweep%d.json" % r)))
        assert tot["device_ms"] == 150.0                 # the slowest rank
        assert tot["evals"] == 1800.0 and tot["neuron_steps"] == 300.0
        assert tot["spikes"] == 9.0 and tot["neurons"] == 30.0


def test_torchrun_reference_arm_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--cpu-sample", "100", "--cpu-ms", "5", "--no-ref-gpu"]
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "1"
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
