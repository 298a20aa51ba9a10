"""Bit-reproducibility across the RK5 kernel variants (needs a B200).

The autotuner picks, by timing, one of NGPU_RK5_VARIANTS kernels for a group
(register caps for 1, 4, 5, 6 and 8 resident blocks per SM, and the
persistent kernel with shared-memory prefetch at 3-6 blocks per SM); with
the straggler queue on or off, and the delivery in the update's grid or on
its own stream. The arithmetic is written with explicit rounding (paired
FP32x2 intrinsics, ex2/lg2/rcp of the special-function unit), so every
choice, and the kernels that integrate several steps per launch, must give
the same state bit for bit: two runs on two machines agree whatever the
timings made the tuner choose.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_VARIANTS = 9


def _run(ngpu, env):
    keys = ("NGB200_RK5_VARIANT", "NGB200_RK5_QUEUE", "NGB200_FUSE_DELIVERY", "NGB200_WINDOW")
    old = {k: os.environ.get(k) for k in keys}
    for k in keys:
        os.environ.pop(k, None)
    os.environ.update(env)
    try:
        b = ngpu.default_binding()
        b.Reset()
        b.SetVerbosityLevel(0)
        ngpu.SetKernelStatus("rnd_seed", 4242)
        pg = ngpu.Create("poisson_generator")
        ngpu.SetStatus(pg, "rate", 20000.0)
        nrn = ngpu.Create("aeif_cond_beta", 20000, 2)
        ngpu.SetStatus(nrn, {"E_rev": [0.0, -85.0], "tau_rise": [0.2, 0.5],
                             "tau_decay": [2.0, 8.0]})
        ngpu.SetNeuronGroupParam(nrn, "rk5_eps", 1e-3)
        ngpu.Connect(pg, nrn, {"rule": "all_to_all"},
                     {"weight": 0.5, "delay": 0.1, "receptor": 0})
        ngpu.Connect(nrn[0:16000], nrn, {"rule": "fixed_indegree", "indegree": 80},
                     {"weight": 0.05, "delay": 1.0, "receptor": 0})
        ngpu.Connect(nrn[16000:20000], nrn, {"rule": "fixed_indegree", "indegree": 20},
                     {"weight": 0.35, "delay": 1.0, "receptor": 1})
        ngpu.ActivateSpikeCount(nrn)
        ngpu.Simulate(60.0)
        tuned = b.GetRk5Tuning(nrn.i0)[0]
        state = [np.asarray(ngpu.GetNeuronVar(nrn.i0, nrn.n, v), dtype=np.float32).view(np.int32)
                 for v in ("V_m", "w", "g", "g1")]
        counts = ngpu.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count")
        return tuned, state, counts
    finally:
        for k in keys:
            if old[k] is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = old[k]


def test_rk5_variants_bit_identical(ngpu):
    ref_v, ref_state, ref_counts = _run(ngpu, {"NGB200_RK5_VARIANT": "0", "NGB200_WINDOW": "0"})
    assert ref_v == 0
    assert ref_counts.sum() > 1000          # the network fires: stragglers exist
    runs = [{"NGB200_RK5_VARIANT": str(v), "NGB200_WINDOW": "0"} for v in range(1, N_VARIANTS)]
    runs += [{"NGB200_RK5_VARIANT": "2", "NGB200_RK5_QUEUE": "0", "NGB200_WINDOW": "0"},
             {"NGB200_RK5_VARIANT": "2", "NGB200_FUSE_DELIVERY": "0", "NGB200_WINDOW": "0"}]
    # several steps per launch (windows of up to 11 steps at 1 ms delays),
    # with the window kernel's register caps
    runs += [{"NGB200_RK5_VARIANT": v} for v in ("0", "1", "2", "3", "6")]
    for env in runs:
        v, state, counts = _run(ngpu, env)
        assert v == int(env["NGB200_RK5_VARIANT"]), env
        assert np.array_equal(counts, ref_counts), env
        for a, b in zip(state, ref_state):
            assert np.array_equal(a, b), env
