"""Multi-process paths of bench.py on the CPU (gloo, world size 2): the
replicas' host-side barrier and max-over-ranks reduction, and a full
torchrun launch of the reference arm in which rank 0 alone prints the JSON
line and every rank exits 0."""
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


def test_torchrun_reference_arm_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--cpu-sample", "100", "--cpu-ms", "5"]
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "1"
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
