"""Times the reference's own CUDA build (oracle/_ref/libneurongpu_ref.so) on
the GPU, driven through its stock C ABI (`src/neurongpu_C.h`), for the
workloads bench.py measures. Test infrastructure only (the reference
baseline); the product never loads that library.

The library keeps one global simulator per process (src/neurongpu_C.cpp:26),
so every run is its own process. The RK5 tolerance of the reference is the
device constant of src/rk5.cu:55 (1e-6); oracle/ref_harness.cu sets it for
the runs at the workloads' 1e-3 and the output says which value ran.

Usage: python oracle/ref_gpu.py [--n N] [--steps K] [--warmup W]
           [--step-ms MS] [--eps 1e-3,1e-6] [--w-pg W]
Prints one JSON object.
"""
import argparse
import ctypes
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "_ref", "libneurongpu_ref.so")


def run(n, steps, warmup, step_ms, eps_list, w_pg=None):
    sys.path.insert(0, ROOT)
    import bench
    from neurongpu_b200 import neurongpu as ngpu_mod
    if not os.path.exists(LIB):
        return {"impl": "reference_gpu", "unavailable": "oracle/_ref/libneurongpu_ref.so not built"}
    b = ngpu_mod.Binding(LIB)
    if b.has_extensions:
        raise RuntimeError("%s is not the reference build" % LIB)
    lib = ctypes.CDLL(LIB)
    lib.NGB200REF_SetRk5Eps.argtypes = [ctypes.c_float]
    lib.NGB200REF_SetRk5Eps.restype = ctypes.c_int
    lib.NGB200REF_GetRk5Eps.restype = ctypes.c_float
    cfg = dict(bench.SCALE)
    cfg["n"] = n
    if w_pg:
        cfg["w_pg"] = w_pg
    b.SetVerbosityLevel(0)
    t0 = time.perf_counter()
    pg, nrn = bench.build_network(b, cfg, eps_param=False)
    b.ActivateSpikeCount(nrn)
    connect_s = time.perf_counter() - t0
    b.Calibrate()
    build_s = time.perf_counter() - t0
    runs = []
    for eps in eps_list:
        if lib.NGB200REF_SetRk5Eps(ctypes.c_float(eps)) != 0:
            raise RuntimeError("could not set the reference RK5 tolerance")
        eps_dev = float(lib.NGB200REF_GetRk5Eps())
        for _ in range(warmup):
            b.Simulate(step_ms)
        c0 = sum(b.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count"))
        t1 = time.perf_counter()
        for _ in range(steps):
            b.Simulate(step_ms)
        wall = time.perf_counter() - t1
        c1 = sum(b.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count"))
        bio = steps * step_ms / 1000.0
        runs.append({"rk5_eps": eps_dev, "bio_s_per_wall_s": bio / wall,
                     "mean_rate_hz": (c1 - c0) / (n * bio),
                     "wall_s_per_bio_s": wall / bio, "timed_bio_s": bio, "wall_s": wall,
                     "eps_source": "src/rk5.cu:55 default" if abs(eps_dev - 1e-6) < 1e-12
                     else "set through oracle/ref_harness.cu"})
    return {"impl": "reference_gpu", "library": "oracle/_ref/libneurongpu_ref.so (reference sources, "
            "nvcc sm_100a, --maxrregcount=55, -rdc)",
            "workload": "scale: %d aeif_cond_beta x %d synapses, Poisson %.0f Hz w %g nS, dt 0.1 ms"
            % (n, cfg["k_exc"] + cfg["k_inh"], cfg["rate"], cfg["w_pg"]),
            "timing": "wall clock around Simulate (the reference's Simulate returns after the "
                      "device work)",
            "connect_s": connect_s, "build_s": build_s, "step_ms": step_ms, "steps": steps,
            "warmup": warmup, "runs": runs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--step-ms", type=float, default=100.0)
    ap.add_argument("--eps", default="1e-3,1e-6")
    ap.add_argument("--w-pg", type=float, default=0.0)
    a = ap.parse_args()
    out = run(a.n, a.steps, a.warmup, a.step_ms, [float(x) for x in a.eps.split(",")], a.w_pg)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
