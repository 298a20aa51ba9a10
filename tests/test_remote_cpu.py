"""Host side of a network partitioned over hosts, on the CPU (gloo, world
size 2): the Python layer's Simulate of a partitioned network runs steps in
runs of the shortest remote delay (the minimum over the hosts), packs each
host's exported spikes, all-gathers the lists and hands every other host's
list to the unpack, growing the pack buffer when a list does not fit. The
library calls are replaced by a recording fake (the kernels themselves are
tested on the GPU, tests/test_gpu_remote.py)."""
import ctypes
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_binding_class():
    sys.path.insert(0, ROOT)
    from neurongpu_b200 import neurongpu as ngpu

    class FakeBinding(ngpu.Binding):
        """Binding whose library calls are recorded: host h emits, in the
        run of steps that starts at step t, 5000 h + t % 7 spikes of
        exported nodes (enough on host 1 to overflow the first buffer)."""

        def __init__(self, comm, e_steps):
            self._comm, self._xbuf = comm, None
            self.e_steps, self.t, self.runs, self.received = e_steps, 0, [], []

        def _call(self, name, *args):
            if name == "NGB200_RemoteExchangeSteps":
                return self.e_steps
            if name == "NGB200_SimulateSteps":
                k = int(args[0].value)
                self.runs.append(k)
                self.t += k
            return 0

        def SetSimTime(self, t):
            return 0

        def GetTimeResolution(self):
            return 0.1

        def _spikes(self):
            h = self._comm.rank
            n = 5000 * h + (self.t % 7)
            return [(j % self.runs[-1], 1000 * h + j, h + 0.5) for j in range(n)]

        def PackRemoteSpikes(self, n_steps, ptr, cap):
            sp = self._spikes()
            words = (ctypes.c_int32 * (4 + 3 * cap)).from_address(ptr)
            for j, (k, node, hgt) in enumerate(sp[:cap]):
                words[4 + 3 * j] = k
                words[5 + 3 * j] = node
                words[6 + 3 * j] = ctypes.c_int32.from_buffer(ctypes.c_float(hgt)).value
            return len(sp)

        def UnpackRemoteSpikes(self, src, n_steps, ptr, count):
            words = (ctypes.c_int32 * (4 + 3 * count)).from_address(ptr)
            first = (words[4], words[5])
            last = (words[4 + 3 * (count - 1)], words[5 + 3 * (count - 1)])
            self.received.append((self.t, src, n_steps, count, first, last))
            return 0

    return FakeBinding


def _worker(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo")
    sys.path.insert(0, ROOT)
    from neurongpu_b200 import neurongpu as ngpu
    comm = ngpu.HostComm()
    fake = _fake_binding_class()(comm, e_steps=(7 if rank == 0 else 5))
    fake._simulate_partitioned(2.3)             # 23 steps
    with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
        f.write(repr({"runs": fake.runs, "received": fake.received}))
    dist.destroy_process_group()


def test_partitioned_simulate_exchanges_every_run(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    out = [eval(open(tmp_path / ("rank%d.txt" % r)).read()) for r in range(2)]
    for r in range(2):
        # runs of the shorter of the two hosts' intervals, then the rest
        assert out[r]["runs"] == [5, 5, 5, 5, 3]
        rec = out[r]["received"]
        assert len(rec) == 5
        other = 1 - r
        t = 0
        for (t_end, src, n_steps, count, first, last), k in zip(rec, out[r]["runs"]):
            t += k
            assert t_end == t and src == other and n_steps == k
            # the other host's whole list arrived, the overflowed first
            # buffer included (host 1: 5000+ spikes against a first buffer of 4096)
            assert count == 5000 * other + (t % 7)
            if count:
                assert first == (0, 1000 * other)
                assert last == ((count - 1) % k, 1000 * other + count - 1)
