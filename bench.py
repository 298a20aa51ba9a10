"""Benchmark of the per-time-step simulation core.

Workload (the scale configuration): 1,000,000 aeif_cond_beta neurons with 2
receptor ports (exc / inh), 80 % excitatory, fixed in-degree 1000 (800 exc,
w = 0.05 nS, port 0; 200 inh, w = 0.35 nS, port 1) = 1e9 synapses with
integer delays of 1-5 ms, an independent 20 kHz Poisson drive per neuron
(w = 0.05 nS), dt = 0.1 ms, RK5 tolerance 1e-3, FP32 state. Synthetic
network generated from a seed; no external data.

A "step" of this benchmark is --step-ms of biological time (default 100 ms =
1000 integration steps). The metric is biological seconds simulated per
wall-clock second (device time of the step loops, CUDA events on the
simulation stream, max over ranks); synaptic events per second are reported
beside it. Multi-GPU runs are independent replicas (weak scaling).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE = dict(n=1_000_000, k_exc=800, k_inh=200, w_exc=0.05, w_inh=0.35, delays=(1, 2, 3, 4, 5),
             rate=20000.0, w_pg=0.05, eps=1e-3)
SMALL = dict(n=1000, k_exc=80, k_inh=20, w_exc=0.05, w_inh=0.35, delays=(1, 2),
             rate=20000.0, w_pg=0.05, eps=1e-3)
NEURON_PARAMS = {"C_m": 281.0, "g_L": 30.0, "E_L": -70.6, "V_th": -50.4, "Delta_T": 2.0,
                 "a": 4.0, "b": 80.5, "tau_w": 144.0, "V_reset": -60.0,
                 "E_rev": [0.0, -85.0], "tau_rise": [0.2, 0.5], "tau_decay": [2.0, 8.0]}
BYTES_PER_NEURON_STEP = 72     # algorithmic: state r+w, h r+w, port inputs
BYTES_PER_EVENT = 8            # algorithmic: 4 B target slot + 4 B weight


def build_network(ngpu, cfg, seed=1234, eps_param=True):
    """The scale network through the drop-in API. Delays are drawn per
    connection group: for every delay value d in 1..5 ms each neuron gets
    k_exc/5 excitatory and k_inh/5 inhibitory inputs, i.e. the integer
    delays are uniform over the 5 values. eps_param: set the RK5 tolerance
    as the group parameter rk5_eps (a library whose tolerance is a fixed
    constant, as the reference's, is given it otherwise)."""
    ngpu.SetKernelStatus("rnd_seed", seed)
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", cfg["rate"])
    n = cfg["n"]
    nrn = ngpu.Create("aeif_cond_beta", n, 2)
    ngpu.SetStatus(nrn, NEURON_PARAMS)
    if eps_param:
        ngpu.SetNeuronGroupParam(nrn, "rk5_eps", cfg["eps"])
    ne = int(0.8 * n)
    exc, inh = nrn[0:ne], nrn[ne:n]
    nd = len(cfg["delays"])
    for d in cfg["delays"]:
        ngpu.Connect(exc, nrn, {"rule": "fixed_indegree", "indegree": cfg["k_exc"] // nd},
                     {"weight": cfg["w_exc"], "delay": float(d), "receptor": 0})
        ngpu.Connect(inh, nrn, {"rule": "fixed_indegree", "indegree": cfg["k_inh"] // nd},
                     {"weight": cfg["w_inh"], "delay": float(d), "receptor": 1})
    ngpu.Connect(pg, nrn, {"rule": "all_to_all"},
                 {"weight": cfg["w_pg"], "delay": 0.1, "receptor": 0})
    return pg, nrn


class ClockSampler(object):
    """nvidia-smi clock / throttle samples during the timed region: started
    before it (nvidia-smi takes a moment to start), every 50 ms; only the
    samples that arrive after mark() count."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.t_mark = 0.0

    def mark(self):
        self.t_mark = time.monotonic()

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, ln in list(self.lines):
            if t < self.t_mark:
                continue
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = max(smax, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM traffic and executed instructions per unit, from ncu captures of the
# same kernels (dram__bytes_read.sum + dram__bytes_write.sum and
# smsp__inst_executed.sum per launch, divided by the neurons / warps / events
# of the launch): the RK5 update (6-blocks/SM variant with the fused
# delivery) on the silent 1e6-neuron network in steady state, caches kept
# between launches (profiles/rk5_update_steady_1m.md); the delivery on the
# active network at 400,000 neurons (profiles/deliver_active_400k.md).
TRAFFIC_RK5_PER_NEURON_STEP = 6.2        # bytes (the state stays L2-resident)
TRAFFIC_DELIVER_PER_EVENT = 11.3         # bytes
# the delivery before a window (k_deliver_window) on the active network at
# 400,000 neurons in windows of 10 steps (profiles/deliver_window_400k.md)
TRAFFIC_DELIVER_WINDOW_PER_EVENT = 20.7  # bytes
INST_RK5_PER_WARP_STEP = 821.9           # warp instructions per 32 neuron-steps
# the window kernel (several steps per launch; register cap for 6 blocks per
# SM), 200,000 neurons of the silent network, windows of 10 steps
# (profiles/rk5_window_200k.md)
TRAFFIC_RK5_WINDOW_PER_NEURON_STEP = 3.69
INST_RK5_WINDOW_PER_WARP_STEP = 634.6
# algorithmic bytes of a window launch per neuron: the state (variables,
# step size, time offset, refractory counter) read and written once per
# window, the port inputs read and cleared every step
BYTES_WINDOW_STATE_PER_NEURON = 56
BYTES_WINDOW_INPUT_PER_NEURON_STEP = 16
SM_COUNT, SMSP_PER_SM = 148, 4


def issue_roofline(n, avg_ms, clocks, steps_per_launch=1, inst_per_warp_step=None):
    """Instruction-issue roofline of the RK5 update (the binding one: the
    kernel issues 650-820 warp instructions per 32 neuron-steps and reads
    its state mostly from L2): warp instructions per launch from the ncu
    count per warp-step, against one instruction per cycle per SM
    sub-partition at the median SM clock sampled during the timed region."""
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    per = INST_RK5_PER_WARP_STEP if inst_per_warp_step is None else inst_per_warp_step
    inst = per * ((n + 31) // 32) * steps_per_launch
    achieved = inst / (avg_ms / 1000.0) / 1e9
    peak = SM_COUNT * SMSP_PER_SM * mhz * 1e6 / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "Ginst/s", "frac": achieved / peak,
            "inst_per_launch": inst, "sm_mhz": mhz}


SAMPLE_VARS = ("V_m", "w", "g", "g1")


def sample_state(ngpu, nrn, idx):
    """State of the sampled neurons (group-local indices idx): V_m, w and
    per port g, g1."""
    import numpy as np
    nodes = [nrn[int(i)] for i in idx]
    out = {}
    for v in SAMPLE_VARS:
        out[v] = np.asarray(ngpu.GetNeuronPtVar(nodes, v), dtype=np.float64).reshape(len(idx), -1)
    return out


def oracle_replay(cfg, idx, n_steps, gpu_state, threads=0):
    """Error of the GPU run against the FP64 oracle: the sampled neurons of
    the silent network (checked by the caller: no spike in the whole run, so
    each neuron saw only its own Poisson drive) replayed for the same number
    of steps with the same random streams; returns the largest deviations
    of the final state."""
    import numpy as np
    from oracle import oracle as orc
    orc.set_threads(threads if threads > 0 else (os.cpu_count() or 1))
    n = len(idx)
    net = orc.Network(dt=0.1, seed=1234)
    net.create(orc.POISSON_GENERATOR, 1, params={"rate": cfg["rate"]})
    p = {k: (np.float32(v) if np.isscalar(v) else [np.float32(x) for x in v])
         for k, v in NEURON_PARAMS.items()}
    grp = net.create(orc.AEIF_COND_BETA, n, 2, params=p, eps=cfg["eps"])
    net.connect(np.zeros(n, dtype=np.int32), np.arange(n) + 1, 0, cfg["w_pg"], 0.1)
    net.set_direct_streams(np.asarray(idx, dtype=np.uint64))
    t0 = time.perf_counter()
    left = n_steps
    while left > 0:
        k = min(left, 10000)
        net.simulate(k)
        left -= k
    wall = time.perf_counter() - t0
    # the GPU's variable getters fold the last step's pending input first
    net.flush()
    nv = len(grp.var_names)
    err = {"V_m_max_abs_mV": 0.0, "V_m_max_rel": 0.0, "w_max_abs_pA": 0.0,
           "g_max_rel": 0.0}
    for k in range(n):
        v, _ = net.state(1 + k, nv)
        dv = abs(v[grp.var_index("V_m")] - gpu_state["V_m"][k, 0])
        err["V_m_max_abs_mV"] = max(err["V_m_max_abs_mV"], dv)
        err["V_m_max_rel"] = max(err["V_m_max_rel"], dv / 70.0)
        err["w_max_abs_pA"] = max(err["w_max_abs_pA"],
                                  abs(v[grp.var_index("w")] - gpu_state["w"][k, 0]))
        for q in range(2):
            for name in ("g", "g1"):
                o = v[grp.var_index(name, q)]
                g = gpu_state[name][k, q]
                err["g_max_rel"] = max(err["g_max_rel"], abs(o - g) / max(abs(o), 1e-3))
    err.update({"neurons": n, "steps": n_steps, "replay_wall_s": wall,
                "against": "FP64 oracle, same Poisson streams, final state of the run"})
    return err


def cpu_baseline(cfg, n_sample=2000, sim_ms=20.0, threads=0):
    """FP64 CPU oracle on a bounded sample of the workload: n_sample neurons
    with the same in-degree, rates and delays, sim_ms of biological time.
    Returns bio-s per wall-s scaled to the full network size (cost linear in
    the number of neurons at fixed in-degree)."""
    import numpy as np
    from oracle import oracle as orc
    orc.set_threads(threads if threads > 0 else (os.cpu_count() or 1))
    threads = orc.get_threads()
    rng = np.random.default_rng(1234)
    n = n_sample
    ne = int(0.8 * n)
    net = orc.Network(dt=0.1, seed=1234)
    net.create(orc.POISSON_GENERATOR, 1, params={"rate": cfg["rate"]})
    p = {k: (np.float32(v) if np.isscalar(v) else [np.float32(x) for x in v])
         for k, v in NEURON_PARAMS.items()}
    net.create(orc.AEIF_COND_BETA, n, 2, params=p, eps=cfg["eps"])
    net.connect(np.zeros(n, dtype=np.int32), np.arange(n) + 1, 0, cfg["w_pg"], 0.1)
    nd = len(cfg["delays"])
    ke, ki = min(cfg["k_exc"], ne) // nd, min(cfg["k_inh"], n - ne) // nd
    for d in cfg["delays"]:
        src = np.concatenate([rng.choice(ne, size=ke, replace=False) for _ in range(n)])
        net.connect(src + 1, np.repeat(np.arange(n) + 1, ke), 0, cfg["w_exc"], float(d))
        src = np.concatenate([ne + rng.choice(n - ne, size=ki, replace=False) for _ in range(n)])
        net.connect(src + 1, np.repeat(np.arange(n) + 1, ki), 1, cfg["w_inh"], float(d))
    steps = int(round(sim_ms / 0.1))
    net.simulate(1)             # builds the oracle's connection tables (untimed)
    t0 = time.perf_counter()
    net.simulate(steps)
    wall = time.perf_counter() - t0
    bio = sim_ms / 1000.0
    value = bio / wall * (n / cfg["n"])
    sample = ("FP64 oracle, %d neurons x in-degree %d, %.0f ms bio, %.2f s wall, "
              "scaled by %d/%d neurons" % (n, ke * nd + ki * nd, sim_ms, wall, n, cfg["n"]))
    return {"value": value, "unit": "bio_s/wall_s", "cores": threads, "kind": "port",
            "sample": sample}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def reduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, world, rank):
    """Reference arm: the reference's own implementation of the path. The
    reference has no CPU implementation of the simulation core; its CUDA
    build (oracle/_ref) is used when it was built, otherwise the FP64 CPU
    restatement (oracle port) on a bounded sample of the same workload."""
    cfg = SCALE if args.config == "scale" else SMALL
    if rank != 0:
        return 0
    metric = "bio_s_per_wall_s"
    vals = []
    for _ in range(max(1, args.warmup)):
        cpu_baseline(cfg, n_sample=args.cpu_sample, sim_ms=5.0)
    for _ in range(args.steps):
        vals.append(cpu_baseline(cfg, n_sample=args.cpu_sample, sim_ms=args.cpu_ms))
    v = sum(x["value"] for x in vals) / len(vals)
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"impl": "reference", "metric": metric, "value": v, "unit": "bio_s/wall_s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "scale: 1M aeif_cond_beta x 1000 synapses, Poisson 20 kHz, "
                                   "dt 0.1 ms, RK5 eps 1e-3", "sample": cb["sample"]},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "bio_s/wall_s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_gpu": reference_gpu(cfg, args)}
    print(json.dumps(line))
    return 0


def reference_gpu(cfg, args):
    """The reference's own CUDA build (oracle/_ref, compiled from its sources
    for sm_100a) on the same workload and GPU, driven through its C ABI in a
    separate process (oracle/ref_gpu.py): wall time of Simulate at the
    workload's RK5 tolerance 1e-3 and at the reference's built-in 1e-6."""
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "libneurongpu_ref.so")
    if not os.path.exists(ref_lib):
        return {"unavailable": "oracle/_ref/libneurongpu_ref.so was not built"}
    if args.no_ref_gpu:
        return {"unavailable": "skipped (--no-ref-gpu)"}
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "ref_gpu.py"), "--n", str(cfg["n"]),
           "--steps", "3", "--warmup", "1", "--step-ms", "100", "--eps", "1e-3,1e-6",
           "--w-pg", str(cfg["w_pg"])]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        return json.loads(r.stdout.strip().split("\n")[-1])
    except Exception as e:
        return {"unavailable": "reference GPU run failed: %s" % str(e)[:200]}


def shard_networks(sizes, world):
    """Independent networks to ranks, greedily by neuron count: the largest
    unassigned network goes to the rank with the fewest neurons so far
    (ties to the lower rank). Returns the network indices of every rank."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += sizes[i]
    return [sorted(x) for x in out]


def reduce_sum(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def sweep_phase_totals(local, world):
    """Whole-sweep figures of one phase from every rank's own: device time is
    the slowest rank's, counts are summed."""
    out = {"device_ms": reduce_max(local["device_ms"], world)}
    for k in ("evals", "spikes", "neuron_steps", "neurons"):
        out[k] = reduce_sum(local[k], world)
    return out


def run_sweep(args, world, rank):
    """Batched + learned workload: 256 independent AdEx networks (sizes
    log-uniform in 1k-50k, in-degree 100-500, a, b and Poisson rate on a
    seeded grid), all RK5 groups of a rank integrated by one batched launch
    per step. With N ranks the networks are sharded by size (no exchange:
    they are independent); the device time is the slowest rank's.
    Phases: plain controller with accepted-step logging, GPU training of the
    step proposer, then the same networks continued with the plain and with
    the learned controller; prints one JSON line comparing them."""
    from tests import sweep
    from neurongpu_b200 import neurongpu as ngpu
    b = ngpu.default_binding()
    b.SetVerbosityLevel(0)
    if args.no_batch:
        b.SetRk5Batching(False)
    grid = sweep.sweep_grid(args.nets, 1000, 50000, 100, 500, seed=2024)
    mine = shard_networks([p["n"] for p in grid], world)[rank]
    my_grid = [grid[i] for i in mine]
    t0 = time.perf_counter()
    nets = sweep.build_sweep(b, my_grid, w_pg=args.sweep_w_pg)
    ngpu.Calibrate()
    build_s = reduce_max(time.perf_counter() - t0, world)
    n_mine = sum(p["n"] for p in my_grid)
    n_tot = sum(p["n"] for p in grid)
    b.SetStepLog(None, args.log_cap)
    b.Simulate(args.step_ms)
    logged = reduce_sum(b.GetStepLogCount(None), world)
    t1 = time.perf_counter()
    rows, l0, l1 = b.TrainStepProposer(steps=args.train_steps, blocks=64, lr=3e-3, seed=5)
    train_s = reduce_max(time.perf_counter() - t1, world)

    def phase():
        e0, s0, ms = b.StageEvaluations(), b.TotalSpikes(), 0.0
        barrier(world)
        for _ in range(args.steps):
            b.Simulate(args.step_ms)
            ms += b.LastSimulateDeviceMs()
        steps = args.steps * args.step_ms / 0.1
        tot = sweep_phase_totals({"device_ms": ms, "evals": b.StageEvaluations() - e0,
                                  "spikes": b.TotalSpikes() - s0,
                                  "neuron_steps": n_mine * steps, "neurons": n_mine}, world)
        bio = args.steps * args.step_ms / 1000.0
        return {"bio_s_per_wall_s": bio / (tot["device_ms"] / 1000.0),
                "device_ms": tot["device_ms"],
                "stage_evals_per_neuron_step": tot["evals"] / tot["neuron_steps"],
                "mean_rate_hz": tot["spikes"] / (tot["neurons"] * bio)}
    for _ in range(args.warmup):
        b.Simulate(args.step_ms)
    plain = phase()
    b.SetStepProposer(None, True)
    for _ in range(args.warmup):
        b.Simulate(args.step_ms)
    learned = phase()
    if rank != 0:
        return 0
    line = {"metric": "sweep_bio_s_per_wall_s", "value": plain["bio_s_per_wall_s"],
            "unit": "bio_s/wall_s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "sweep: %d aeif_cond_beta networks, %d neurons, sizes "
                                   "log-uniform 1k-50k, in-degree 100-500, a 0-8 nS, b 0-150 pA, "
                                   "Poisson 10-30 kHz w %g nS, dt 0.1 ms, RK5 eps 1e-3"
                                   % (len(grid), n_tot, args.sweep_w_pg),
                       "batched_launch": not args.no_batch, "step_bio_ms": args.step_ms,
                       "parallelism": ("networks sharded by size over %d ranks, no exchange"
                                       % world) if world > 1 else "single"},
            "build_s": build_s, "logged_substeps": logged, "train_rows": rows,
            "train_loss_first": l0, "train_loss_last": l1, "train_s": train_s,
            "plain": plain, "learned": learned,
            "stage_eval_reduction": 1.0 - learned["stage_evals_per_neuron_step"]
            / plain["stage_evals_per_neuron_step"],
            "rk5_tuning": b.GetRk5Tuning(nets[0].i0)}
    print(json.dumps(line))
    return 0


def run_network(ngpu, b, cfg, args, world, step_ms, steps, warmup):
    """Builds the network of cfg, warms up, then measures: the timed region
    (device time of the step loops, no instrumentation), a second run of the
    same length with CUDA events around every kernel class (per-kernel
    launch durations), and the counters. Returns a dict."""
    t_build = time.perf_counter()
    pg, nrn = build_network(ngpu, cfg)
    ngpu.ActivateSpikeCount(nrn)
    connect_s = time.perf_counter() - t_build
    ngpu.Calibrate()
    build_s = time.perf_counter() - t_build
    sampler = ClockSampler(0)
    sampler.start()
    for _ in range(warmup):
        ngpu.Simulate(step_ms)
    ev0, evals0, spikes0 = b.DeliveredEvents(), b.StageEvaluations(), b.TotalSpikes()
    barrier(world)
    sampler.mark()
    dev_ms = 0.0
    for _ in range(steps):
        ngpu.Simulate(step_ms)
        dev_ms += b.LastSimulateDeviceMs()
    clocks = sampler.stop()
    barrier(world)
    dev_ms_max = reduce_max(dev_ms, world)
    r = {"pg": pg, "nrn": nrn, "build_s": build_s, "connect_s": connect_s, "clocks": clocks,
         "dev_ms": dev_ms_max, "kernels_per_step": b.KernelsPerStep(),
         "events": b.DeliveredEvents() - ev0, "evals": b.StageEvaluations() - evals0,
         "spikes": b.TotalSpikes() - spikes0, "steps_run": warmup + steps}
    # the same steps with events around every kernel class (serial delivery)
    b.SetKernelTiming(True)
    ev1 = b.DeliveredEvents()
    for _ in range(steps):
        ngpu.Simulate(step_ms)
    r["events_instr"] = b.DeliveredEvents() - ev1
    r["ktime"] = {k: b.GetKernelTiming(i) for i, k in
                  enumerate(("update", "deliver", "stdp", "bookkeeping"))}
    b.SetKernelTiming(False)
    r["steps_run"] += steps
    r["tuning"] = b.GetRk5Tuning(nrn.i0)
    return r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--config", default="scale", choices=["scale", "small", "sweep"])
    ap.add_argument("--nets", type=int, default=256, help="sweep: number of networks")
    ap.add_argument("--sweep-w-pg", type=float, default=0.2, help="sweep: Poisson weight (nS)")
    ap.add_argument("--log-cap", type=int, default=65536, help="sweep: logged sub-steps per group")
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--no-batch", action="store_true", help="sweep: one RK5 launch per network")
    ap.add_argument("--step-ms", type=float, default=100.0)
    ap.add_argument("--cpu-sample", type=int, default=16000)
    ap.add_argument("--cpu-ms", type=float, default=100.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip the reference's CUDA build")
    ap.add_argument("--no-active", action="store_true",
                    help="skip the active (26 Hz) variant of the workload")
    ap.add_argument("--active-w-pg", type=float, default=0.5,
                    help="Poisson weight (nS) of the active variant")
    ap.add_argument("--n", type=int, default=0, help="override the number of neurons")
    ap.add_argument("--k-in", type=int, default=0,
                    help="override the in-degree (80 %% exc / 20 %% inh; profiling captures "
                         "of the update kernel at a small device footprint)")
    ap.add_argument("--w-pg", type=float, default=0.0,
                    help="override the Poisson drive weight (nS) for an active network")
    args = ap.parse_args()
    if args.n > 0:
        SCALE["n"] = SMALL["n"] = args.n
    if args.k_in > 0:
        for c in (SCALE, SMALL):
            c["k_exc"], c["k_inh"] = (4 * args.k_in) // 5, args.k_in // 5
    if args.w_pg > 0:
        SCALE["w_pg"] = SMALL["w_pg"] = args.w_pg
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    os.environ.setdefault("CUDA_VISIBLE_DEVICES", str(local))
    if args.config == "sweep":
        return run_sweep(args, world, rank)
    import numpy as np
    cfg = SCALE if args.config == "scale" else SMALL
    from neurongpu_b200 import neurongpu as ngpu
    b = ngpu.default_binding()
    b.SetVerbosityLevel(0)
    step_ms = args.step_ms
    r = run_network(ngpu, b, cfg, args, world, step_ms, args.steps, args.warmup)
    pg, nrn = r["pg"], r["nrn"]
    bio_s = args.steps * step_ms / 1000.0
    dev_ms_max = r["dev_ms"]
    value = world * bio_s / (dev_ms_max / 1000.0)
    n_steps = int(round(args.steps * step_ms / 0.1))
    step_launch_ms = dev_ms_max / n_steps
    upd_ms, upd_n = r["ktime"]["update"]
    # Roofline of the RK5 update from the uninstrumented timed run: with
    # about one launch per step (the update with the delivery in its grid,
    # 1.02 launches per step with the chunk prologue and epilogue) the
    # launch lasts at most the device time per step; with the delivery on
    # its own stream the update's own duration comes from the instrumented
    # run, capped by the step time.
    # With several steps per launch (a quiet network whose delays allow
    # windows) the update launch integrates W steps; its duration comes from
    # the instrumented run's events around it (nothing runs beside it).
    spl = n_steps / max(upd_n, 1)
    window = spl > 1.5
    one_launch = r["kernels_per_step"] <= 1.1
    peak, peak_kind = measured_peaks()
    if window:
        W = int(round(spl))
        avg_ms = upd_ms / max(upd_n, 1)
        bytes_launch = cfg["n"] * (BYTES_WINDOW_STATE_PER_NEURON +
                                   BYTES_WINDOW_INPUT_PER_NEURON_STEP * W)
        iss = issue_roofline(cfg["n"], avg_ms, r["clocks"], W, INST_RK5_WINDOW_PER_WARP_STEP)
        traffic = TRAFFIC_RK5_WINDOW_PER_NEURON_STEP * cfg["n"] * W
        kernel = "rk5_window"
        timing = ("window launch events of the instrumented run (%d integration steps per "
                  "launch)" % W)
    else:
        W = 1
        avg_ms = step_launch_ms if one_launch else min(upd_ms / max(upd_n, 1), step_launch_ms)
        bytes_launch = BYTES_PER_NEURON_STEP * cfg["n"]
        iss = issue_roofline(cfg["n"], avg_ms, r["clocks"])
        traffic = TRAFFIC_RK5_PER_NEURON_STEP * cfg["n"]
        kernel = "rk5_update"
        timing = ("device time per integration step of the uninstrumented timed run "
                  "(%.2f launches per step)" % r["kernels_per_step"]) if one_launch else \
                 "update launch events of a second run, capped by the step time"
    hbm_achieved = bytes_launch / (avg_ms / 1000.0) / 1e9
    roof = {"kernel": kernel, "bound": "issue", "achieved": iss["achieved"],
            "peak": iss["peak"], "unit": "Ginst/s", "frac": iss["frac"],
            "inst_per_launch": iss["inst_per_launch"], "sm_mhz": iss["sm_mhz"],
            "traffic": traffic, "avg_launch_ms": avg_ms, "steps_per_launch": W,
            "timing": timing,
            "hbm": {"achieved": hbm_achieved, "peak": peak, "peak_source": peak_kind,
                    "unit": "GB/s", "frac": hbm_achieved / peak, "traffic": traffic,
                    "bytes_per_launch": bytes_launch},
            "kernel_ms": {k: v[0] for k, v in r["ktime"].items()},
            "launches": {k: v[1] for k, v in r["ktime"].items()}}
    # end-to-end through the public API: H2D of the generator parameters,
    # the simulation call, D2H of the per-neuron spike counts
    def e2e_step():
        ngpu.SetStatus(pg, "rate", cfg["rate"])
        ngpu.Simulate(step_ms)
        return ngpu.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count")
    for _ in range(args.warmup):
        e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_wall = reduce_max(time.perf_counter() - t0, world)
    steps_run = r["steps_run"] + args.warmup + args.steps
    e2e = {"value": world * args.steps * step_ms / 1000.0 / e2e_wall, "unit": "bio_s/wall_s",
           "h2d_bytes_per_step": 48, "d2h_bytes_per_step": 4 * cfg["n"]}
    rate_hz = r["spikes"] / (cfg["n"] * bio_s)
    # final state of a sample of neurons for the error against the oracle
    # (meaningful while the whole run stayed silent)
    silent_run = b.TotalSpikes() == 0
    idx = np.linspace(0, cfg["n"] - 1, min(256, cfg["n"])).astype(np.int64)
    gpu_state = sample_state(ngpu, nrn, idx) if silent_run else None
    line = {
        "metric": "bio_s_per_wall_s", "value": value, "unit": "bio_s/wall_s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": ("scale" if args.config == "scale" else "small")
                   + ": %d aeif_cond_beta x %d synapses, Poisson %.0f Hz w %g nS, dt 0.1 ms, "
                   "RK5 eps %g" % (cfg["n"], cfg["k_exc"] + cfg["k_inh"], cfg["rate"],
                                   cfg["w_pg"], cfg["eps"]),
                   "step_bio_ms": step_ms, "integration_steps": n_steps,
                   "l2": ("no flush: the synapse tables (%.1f GB) exceed L2; the neuron state "
                          "(%d MB) stays L2-resident across the integration steps of a bench "
                          "step, as in any run of the simulator"
                          % (cfg["n"] * (cfg["k_exc"] + cfg["k_inh"]) * 8 / 1e9,
                             cfg["n"] * 72 // 1000000)),
                   "parallelism": "replicas" if world > 1 else "single"},
        "syn_events_per_s": world * r["events"] / (dev_ms_max / 1000.0),
        "mean_rate_hz": rate_hz,
        "rk5_stage_evals_per_neuron_step": r["evals"] / (cfg["n"] * n_steps),
        "wall_per_bio_s": (dev_ms_max / 1000.0) / bio_s,
        "rk5_tuning": r["tuning"],
        "build_s": r["build_s"], "connect_s": r["connect_s"],
        "calibrate_s": r["build_s"] - r["connect_s"],
        "gpu_launches": int(round(r["kernels_per_step"] * n_steps)),
        "roofline": roof,
        "e2e": e2e,
        "clocks": r["clocks"],
    }
    # the same network at a drive that makes it fire (delivery measured)
    if not args.no_active and args.config == "scale":
        acfg = dict(cfg)
        acfg["w_pg"] = args.active_w_pg
        b.Reset()
        b.SetVerbosityLevel(0)
        a_steps = max(1, min(args.steps, 3))
        ar = run_network(ngpu, b, acfg, args, world, step_ms, a_steps, max(1, min(args.warmup, 3)))
        a_bio = a_steps * step_ms / 1000.0
        a_nst = int(round(a_steps * step_ms / 0.1))
        d_ms, d_n = ar["ktime"]["deliver"]
        a_window = a_nst / max(ar["ktime"]["update"][1], 1) > 1.5
        ev_launch = ar["events_instr"] / max(d_n, 1)
        d_avg = d_ms / max(d_n, 1)
        d_ach = BYTES_PER_EVENT * ev_launch / (d_avg / 1000.0) / 1e9 if d_avg > 0 else 0.0
        # the delivery's own bound: its inner loop alone (8 B read and one
        # 64-bit reduction per event into the network's accumulators),
        # measured on this GPU
        try:
            probe = b.StreamingDeliveryRate(2 * acfg["n"], max(1, int(ev_launch)), 10)
        except Exception:
            probe = None
        ev_rate = ev_launch / (d_avg / 1000.0) if d_avg > 0 else 0.0
        line["active"] = {
            "workload": "the same network with Poisson w %g nS" % acfg["w_pg"],
            "value": world * a_bio / (ar["dev_ms"] / 1000.0), "unit": "bio_s/wall_s",
            "ms_per_step": ar["dev_ms"] / a_steps, "steps": a_steps,
            "syn_events_per_s": world * ar["events"] / (ar["dev_ms"] / 1000.0),
            "mean_rate_hz": ar["spikes"] / (acfg["n"] * a_bio),
            "rk5_stage_evals_per_neuron_step": ar["evals"] / (acfg["n"] * a_nst),
            "kernels_per_step": ar["kernels_per_step"],
            "deliver_roofline": {"kernel": "deliver", "bound": "hbm", "achieved": d_ach,
                                 "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                                 "frac": d_ach / peak, "events_per_launch": ev_launch,
                                 "traffic": (TRAFFIC_DELIVER_WINDOW_PER_EVENT if a_window
                                             else TRAFFIC_DELIVER_PER_EVENT) * ev_launch,
                                 "avg_launch_ms": d_avg,
                                 "timing": "delivery launch events of the instrumented run "
                                           + ("(one delivery before each window of steps, "
                                              "one more per chunk)" if a_window
                                              else "(serial delivery)"),
                                 "l2_atomics": None if not probe else {
                                     "achieved": ev_rate, "peak": probe, "unit": "events/s",
                                     "frac": ev_rate / probe,
                                     "peak_source": "measured in this run: the delivery's inner "
                                                    "loop alone on the same events and "
                                                    "accumulators (NGB200_StreamingDeliveryRate)"}},
            "kernel_ms": {k: v[0] for k, v in ar["ktime"].items()},
            "rk5_tuning": ar["tuning"], "clocks": ar["clocks"]}
    if rank != 0:
        barrier(world)
        return 0
    cpu = None
    if not args.no_cpu:
        try:
            cpu = cpu_baseline(cfg, n_sample=args.cpu_sample, sim_ms=args.cpu_ms)
        except Exception as e:
            cpu = {"error": str(e)}
        if gpu_state is not None:
            try:
                line["oracle_err"] = oracle_replay(cfg, idx, steps_run * int(round(step_ms / 0.1)),
                                                   gpu_state)
            except Exception as e:
                line["oracle_err"] = {"error": str(e)[:300]}
        else:
            line["oracle_err"] = {"unavailable": "the network spiked; sampled neurons are not "
                                                 "independent of the rest"}
    line["cpu_baseline"] = cpu
    print(json.dumps(line))
    sys.stdout.flush()
    barrier(world)
    return 0


if __name__ == "__main__":
    sys.exit(main())
