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
    """nvidia-smi clock / throttle samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

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
        for ln in self.lines:
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
# of the launch): RK5 update (8-blocks/SM variant) on the silent network at
# 200,000 neurons in steady state (cold cache; the state's writes stay in L2
# during the launch), delivery on the active network at 400,000 neurons.
TRAFFIC_RK5_PER_NEURON_STEP = 52.4       # bytes
TRAFFIC_DELIVER_PER_EVENT = 11.3         # bytes
INST_RK5_PER_WARP_STEP = 995.2           # warp instructions per 32 neuron-steps
SM_COUNT, SMSP_PER_SM = 148, 4


def issue_roofline(kname, n, avg_ms, clocks):
    """Instruction-issue view of the RK5 update (it is issue and latency
    bound, not HBM bound): warp instructions per launch from the ncu count
    per warp-step, against one instruction per cycle per SM sub-partition at
    the median SM clock sampled during the timed region."""
    if kname != "rk5_update" or avg_ms <= 0:
        return None
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    inst = INST_RK5_PER_WARP_STEP * ((n + 31) // 32)
    achieved = inst / (avg_ms / 1000.0) / 1e9
    peak = SM_COUNT * SMSP_PER_SM * mhz * 1e6 / 1e9
    return {"unit": "Ginst/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "inst_per_launch": inst, "sm_mhz": mhz}


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
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "libneurongpu_ref.so")
    metric = "bio_s_per_wall_s"
    if os.path.exists(ref_lib) and args.ref_gpu:
        line = {"impl": "reference", "unavailable": "reference GPU arm not enabled"}
        print(json.dumps(line))
        return 0
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
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_sweep(args, world, rank):
    """Batched + learned workload: 256 independent AdEx networks (sizes
    log-uniform in 1k-50k, in-degree 100-500, a, b and Poisson rate on a
    seeded grid), all RK5 groups integrated by one batched launch per step.
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
    t0 = time.perf_counter()
    nets = sweep.build_sweep(b, grid, w_pg=args.sweep_w_pg)
    ngpu.Calibrate()
    build_s = time.perf_counter() - t0
    n_tot = sum(p["n"] for p in grid)
    b.SetStepLog(None, args.log_cap)
    b.Simulate(args.step_ms)
    logged = b.GetStepLogCount(None)
    t1 = time.perf_counter()
    rows, l0, l1 = b.TrainStepProposer(steps=args.train_steps, blocks=64, lr=3e-3, seed=5)
    train_s = time.perf_counter() - t1

    def phase():
        e0, s0, ms = b.StageEvaluations(), b.TotalSpikes(), 0.0
        for _ in range(args.steps):
            b.Simulate(args.step_ms)
            ms += b.LastSimulateDeviceMs()
        steps = n_tot * args.steps * args.step_ms / 0.1
        bio = args.steps * args.step_ms / 1000.0
        return {"bio_s_per_wall_s": bio / (ms / 1000.0), "device_ms": ms,
                "stage_evals_per_neuron_step": (b.StageEvaluations() - e0) / steps,
                "mean_rate_hz": (b.TotalSpikes() - s0) / (n_tot * bio)}
    for _ in range(args.warmup):
        b.Simulate(args.step_ms)
    plain = phase()
    b.SetStepProposer(None, True)
    for _ in range(args.warmup):
        b.Simulate(args.step_ms)
    learned = phase()
    line = {"metric": "sweep_bio_s_per_wall_s", "value": plain["bio_s_per_wall_s"],
            "unit": "bio_s/wall_s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "sweep: %d aeif_cond_beta networks, %d neurons, sizes "
                                   "log-uniform 1k-50k, in-degree 100-500, a 0-8 nS, b 0-150 pA, "
                                   "Poisson 10-30 kHz w %g nS, dt 0.1 ms, RK5 eps 1e-3"
                                   % (len(grid), n_tot, args.sweep_w_pg),
                       "batched_launch": not args.no_batch, "step_bio_ms": args.step_ms},
            "build_s": build_s, "logged_substeps": logged, "train_rows": rows,
            "train_loss_first": l0, "train_loss_last": l1, "train_s": train_s,
            "plain": plain, "learned": learned,
            "stage_eval_reduction": 1.0 - learned["stage_evals_per_neuron_step"]
            / plain["stage_evals_per_neuron_step"],
            "rk5_tuning": b.GetRk5Tuning(nets[0].i0)}
    print(json.dumps(line))
    return 0


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
    ap.add_argument("--ref-gpu", action="store_true")
    ap.add_argument("--n", type=int, default=0, help="override the number of neurons")
    ap.add_argument("--w-pg", type=float, default=0.0,
                    help="override the Poisson drive weight (nS) for an active network")
    args = ap.parse_args()
    if args.n > 0:
        SCALE["n"] = SMALL["n"] = args.n
    if args.w_pg > 0:
        SCALE["w_pg"] = SMALL["w_pg"] = args.w_pg
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    os.environ.setdefault("CUDA_VISIBLE_DEVICES", str(local))
    if args.config == "sweep":
        return run_sweep(args, world, rank)
    cfg = SCALE if args.config == "scale" else SMALL
    from neurongpu_b200 import neurongpu as ngpu
    b = ngpu.default_binding()
    b.SetVerbosityLevel(0)
    t_build = time.perf_counter()
    pg, nrn = build_network(ngpu, cfg)
    ngpu.ActivateSpikeCount(nrn)
    connect_s = time.perf_counter() - t_build
    ngpu.Calibrate()
    build_s = time.perf_counter() - t_build
    step_ms = args.step_ms
    # warm-up
    for _ in range(args.warmup):
        ngpu.Simulate(step_ms)
    # timed region (device time of the step loops), per-kernel events on
    # timed region: device time of the step loops (CUDA events on the
    # simulation stream), no per-kernel instrumentation
    ev0 = b.DeliveredEvents()
    evals0 = b.StageEvaluations()
    spikes0 = b.TotalSpikes()
    barrier(world)
    sampler = ClockSampler(0)
    sampler.start()
    dev_ms = 0.0
    for _ in range(args.steps):
        ngpu.Simulate(step_ms)
        dev_ms += b.LastSimulateDeviceMs()
    clocks = sampler.stop()
    barrier(world)
    dev_ms_max = reduce_max(dev_ms, world)
    kernels_per_step = b.KernelsPerStep()
    events = b.DeliveredEvents() - ev0
    evals = b.StageEvaluations() - evals0
    spikes = b.TotalSpikes() - spikes0
    # same number of steps again with CUDA events around every kernel class
    # of every step, for the per-kernel launch durations of the roofline
    b.SetKernelTiming(True)
    ev1 = b.DeliveredEvents()
    for _ in range(args.steps):
        ngpu.Simulate(step_ms)
    events_instr = b.DeliveredEvents() - ev1
    upd_ms, upd_n = b.GetKernelTiming(0)
    del_ms, del_n = b.GetKernelTiming(1)
    stdp_ms, stdp_n = b.GetKernelTiming(2)
    oth_ms, oth_n = b.GetKernelTiming(3)
    b.SetKernelTiming(False)
    bio_s = args.steps * step_ms / 1000.0
    value = world * bio_s / (dev_ms_max / 1000.0)
    events_per_s = world * events / (dev_ms_max / 1000.0)
    n_steps = int(round(args.steps * step_ms / 0.1))
    # roofline of the dominant kernel
    peak, peak_kind = measured_peaks()
    if upd_ms >= del_ms:
        kname = "rk5_update"
        bytes_launch = BYTES_PER_NEURON_STEP * cfg["n"]
        avg_ms = upd_ms / max(upd_n, 1)
        traffic = TRAFFIC_RK5_PER_NEURON_STEP * cfg["n"]
    else:
        kname = "deliver"
        ev_launch = events_instr / max(del_n, 1)
        bytes_launch = BYTES_PER_EVENT * ev_launch
        avg_ms = del_ms / max(del_n, 1)
        traffic = TRAFFIC_DELIVER_PER_EVENT * ev_launch
    achieved = bytes_launch / (avg_ms / 1000.0) / 1e9
    roof = {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak,
            "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "avg_launch_ms": avg_ms,
            "issue": issue_roofline(kname, cfg["n"], avg_ms, clocks),
            "kernel_ms": {"update": upd_ms, "deliver": del_ms, "stdp": stdp_ms,
                          "bookkeeping": oth_ms},
            "launches": {"update": upd_n, "deliver": del_n, "stdp": stdp_n,
                         "bookkeeping": oth_n},
            "timing": "kernel events over a second run of the timed steps"}
    # end-to-end through the public API: H2D of the generator parameters,
    # the simulation call, D2H of the per-neuron spike counts
    # (untimed warm-up first: switching the kernel events off above dropped
    # the captured step graphs)
    def e2e_step():
        ngpu.SetStatus(pg, "rate", cfg["rate"])
        ngpu.Simulate(step_ms)
        return ngpu.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count")
    for _ in range(args.warmup):
        e2e_step()
    e2e_steps = args.steps
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        counts = e2e_step()
    e2e_wall = reduce_max(time.perf_counter() - t0, world)
    e2e = {"value": world * e2e_steps * step_ms / 1000.0 / e2e_wall, "unit": "bio_s/wall_s",
           "h2d_bytes_per_step": 48, "d2h_bytes_per_step": 4 * cfg["n"]}
    rate_hz = spikes / (cfg["n"] * bio_s)
    if rank != 0:
        barrier(world)
        return 0
    cpu = None
    if not args.no_cpu:
        try:
            cpu = cpu_baseline(cfg, n_sample=args.cpu_sample, sim_ms=args.cpu_ms)
        except Exception as e:
            cpu = {"error": str(e)}
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
                   "l2": "inputs larger than L2 (1e9 synapses, 8 GB)",
                   "parallelism": "replicas" if world > 1 else "single"},
        "syn_events_per_s": events_per_s,
        "mean_rate_hz": rate_hz,
        "rk5_stage_evals_per_neuron_step": evals / (cfg["n"] * n_steps),
        "wall_per_bio_s": (dev_ms_max / 1000.0) / bio_s,
        "rk5_tuning": b.GetRk5Tuning(nrn.i0),
        "build_s": build_s, "connect_s": connect_s, "calibrate_s": build_s - connect_s,
        "gpu_launches": int(round(kernels_per_step * n_steps)),
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
    }
    print(json.dumps(line))
    sys.stdout.flush()
    barrier(world)
    return 0


if __name__ == "__main__":
    sys.exit(main())
