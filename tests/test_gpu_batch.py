"""Batched RK5 launches (one kernel per step for many node groups through a
device segment table) against one launch per group. Needs a B200.

Both paths run the same per-neuron arithmetic (the same device function), so
spike trains, state and stage-evaluation counts must be bit-identical for the
same kernel variant. The autotuner is switched off here: its occupancy
variants differ in register allocation, and the compiler may then contract
or schedule floating-point operations differently (last-bit differences).
"""
import os

import numpy as np
import pytest

from tests import sweep

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fixed_variant():
    old = os.environ.get("NGB200_AUTOTUNE")
    os.environ["NGB200_AUTOTUNE"] = "0"
    yield
    if old is None:
        del os.environ["NGB200_AUTOTUNE"]
    else:
        os.environ["NGB200_AUTOTUNE"] = old


def _run(ngpu, batching, grid, t_ms=200.0):
    ngpu.Reset()
    ngpu.SetRk5Batching(batching)
    nets = sweep.build_sweep(ngpu, grid)
    for nrn in nets:
        ngpu.ActivateSpikeCount(nrn)
    ngpu.Simulate(t_ms)
    counts = np.concatenate([ngpu.GetNeuronIntVarArray(n.i0, n.n, "spike_count") for n in nets])
    v = np.concatenate([np.asarray(ngpu.GetNeuronVar(n.i0, n.n, "V_m"), dtype=np.float32).ravel()
                        for n in nets])
    w = np.concatenate([np.asarray(ngpu.GetNeuronVar(n.i0, n.n, "w"), dtype=np.float32).ravel()
                        for n in nets])
    batch_ids = [ngpu.Rk5BatchOf(n.i0) for n in nets]
    return counts, v, w, ngpu.StageEvaluations(), batch_ids


def test_batched_equals_per_group(ngpu):
    grid = sweep.sweep_grid(12, 300, 5000, 50, 150, seed=7)
    c1, v1, w1, e1, b1 = _run(ngpu, True, grid)
    c0, v0, w0, e0, b0 = _run(ngpu, False, grid)
    assert all(b == 0 for b in b1) and all(b == -1 for b in b0)
    assert c1.sum() > 0
    assert np.array_equal(c1, c0)
    assert np.array_equal(v1.view(np.int32), v0.view(np.int32))
    assert np.array_equal(w1.view(np.int32), w0.view(np.int32))
    assert e1 == e0


def test_batched_mixed_models(ngpu):
    """Groups of two models form two batches; a lone group keeps its own
    launch; results equal the unbatched run."""
    def build(batching):
        ngpu.Reset()
        ngpu.SetRk5Batching(batching)
        ngpu.SetKernelStatus("rnd_seed", 3)
        pg = ngpu.Create("poisson_generator")
        ngpu.SetStatus(pg, "rate", 20000.0)
        groups = [ngpu.Create("aeif_cond_beta", 700, 2), ngpu.Create("aeif_cond_alpha", 500, 2),
                  ngpu.Create("aeif_cond_beta", 900, 2), ngpu.Create("aeif_cond_alpha", 300, 2),
                  ngpu.Create("aeif_psc_exp", 400, 2)]
        ngpu.SetStatus(groups[2], {"b": 20.0})
        for g in groups:
            ngpu.Connect(pg, g, {"rule": "all_to_all"}, {"weight": 0.4, "delay": 0.1,
                                                         "receptor": 0})
            ngpu.Connect(g, groups[0], {"rule": "fixed_indegree", "indegree": 20},
                         {"weight": 0.05, "delay": 1.0, "receptor": 0})
            ngpu.ActivateSpikeCount(g)
        ngpu.Simulate(100.0)
        counts = np.concatenate([ngpu.GetNeuronIntVarArray(g.i0, g.n, "spike_count")
                                 for g in groups])
        return counts, [ngpu.Rk5BatchOf(g.i0) for g in groups]
    c1, b1 = build(True)
    c0, b0 = build(False)
    assert b1[0] == b1[2] and b1[1] == b1[3] and b1[0] != b1[1] and b1[4] == -1
    assert c1.sum() > 0
    assert np.array_equal(c1, c0)


def test_straggler_queue_bit_identical(ngpu):
    """Neurons still inside the time step after their first sub-step are
    finished from the straggler queue by a second launch; the result equals
    the uninterrupted loop bit for bit, batched and per group. The update
    kernel runs as its one-block-per-SM variant here, the register budget
    the finishing kernel is compiled for, so both compile the sub-step
    identically."""
    grid = sweep.sweep_grid(12, 300, 5000, 50, 150, seed=7)
    old = {k: os.environ.get(k) for k in ("NGB200_RK5_QUEUE", "NGB200_RK5_VARIANT")}
    res = {}
    try:
        os.environ["NGB200_RK5_VARIANT"] = "0"
        for queue in ("1", "0"):
            os.environ["NGB200_RK5_QUEUE"] = queue
            for batching in (True, False):
                res[(queue, batching)] = _run(ngpu, batching, grid)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    c0, v0, w0, e0, _ = res[("0", False)]
    neuron_steps = sum(p["n"] for p in grid) * 2000
    assert c0.sum() > 0
    assert e0 > 6 * neuron_steps          # some neurons took several sub-steps
    for key, (c, v, w, e, _) in res.items():
        assert np.array_equal(c, c0), key
        assert np.array_equal(v.view(np.int32), v0.view(np.int32)), key
        assert np.array_equal(w.view(np.int32), w0.view(np.int32)), key
        assert e == e0, key


def test_simple_models_batched_equals_per_group(ngpu):
    """The cortical column's eight iaf_psc_exp populations (10 % scale) plus
    groups of iaf_psc_exp_g and izhikevich_psc_exp_2s, updated by one batched
    launch per step, give the same spikes and state as one launch per group."""
    from tests import cortical_column as cc

    def run(batching):
        ngpu.Reset()
        ngpu.SetRk5Batching(batching)
        pops, gens, d = cc.build(ngpu, n_scaling=0.1, k_scaling=0.1, seed=12349)
        izh = ngpu.Create("izhikevich_psc_exp_2s", 500)
        ngpu.SetStatus(izh, {"I_e": 10.0})
        ig = ngpu.Create("iaf_psc_exp_g", 300)
        ngpu.SetStatus(ig, {"I_e": 400.0})
        groups = list(pops) + [izh, ig]
        for p in groups:
            ngpu.ActivateSpikeCount(p)
        ngpu.Simulate(200.0)
        counts = np.concatenate([ngpu.GetNeuronIntVarArray(p.i0, p.n, "spike_count")
                                 for p in groups])
        v = np.concatenate([np.asarray(ngpu.GetNeuronVar(p.i0, p.n, "V_m_rel"),
                                       dtype=np.float32).ravel() for p in pops])
        return counts, v

    c1, v1 = run(True)
    c0, v0 = run(False)
    assert c1.sum() > 100
    assert np.array_equal(c1, c0)
    assert np.array_equal(v1.view(np.int32), v0.view(np.int32))
