"""Network-level parity of the CUDA core with the FP64 oracle. Needs a B200.

Both sides run the same network: it is built once through the drop-in API
(so the connection rules of the library are exercised), every connection is
read back in bulk and loaded into the oracle, and the Poisson input is drawn
from the same counter-based streams, so inputs agree draw by draw. FP32 and
FP64 trajectories separate once the first spike times differ by a step, after
which recurrent networks diverge chaotically; the comparison is therefore
exact early on and statistical afterwards. Tolerances (stated per test):
  * spike trains before divergence: >= 99% of oracle spikes matched by the
    same neuron within one step;
  * population rates: relative difference within the Poisson counting error
    of the population (3 sigma) plus 5%;
  * ISI coefficient-of-variation distributions: two-sample KS p > 1e-3;
  * STDP weights: exact (1e-5) while spike trains agree; afterwards the
    weight histograms (20 bins) within an L1 distance of 0.1 and mean
    weights within 2%.
"""
import numpy as np
import pytest

from tests import cortical_column as cc

pytestmark = pytest.mark.gpu


def _gpu_spikes(ngpu, nodes_first, n_total):
    steps, nodes = [], []
    for i in range(nodes_first, nodes_first + n_total):
        t = ngpu.GetRecSpikeTimes(i)
        if t:
            steps.append(np.rint(np.asarray(t) / 0.1).astype(np.int64) - 1)
            nodes.append(np.full(len(t), i, dtype=np.int64))
    if not steps:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    return np.concatenate(steps), np.concatenate(nodes)


def _match_fraction(o_steps, o_nodes, g_steps, g_nodes, upto):
    gs = {}
    for s, n in zip(g_steps, g_nodes):
        if s < upto + 2:
            gs.setdefault(int(n), []).append(int(s))
    m = o_steps < upto
    tot = int(np.count_nonzero(m))
    hit = 0
    for s, n in zip(o_steps[m], o_nodes[m]):
        if any(abs(int(s) - s2) <= 1 for s2 in gs.get(int(n), [])):
            hit += 1
    return hit, tot


def _pop_bounds(pops):
    return [p.i0 for p in pops], [p.n for p in pops]


def test_cortical_column_scaled_vs_oracle(ngpu):
    """Cortical column at 10% neurons and 10% in-degree (7,717 iaf_psc_exp,
    about 3e6 synapses, fixed_total_number with normal_clipped weights and
    delays), 200 ms settling + 1 s: per-population rates and ISI-CV
    distributions against the oracle; early spike trains identical."""
    from scipy import stats
    seed = 12349
    pops, gens, d = cc.build(ngpu, n_scaling=0.1, k_scaling=0.1, seed=seed)
    first, sizes = _pop_bounds(pops)
    n_total = int(sum(sizes))
    for p in pops:
        ngpu.ActivateRecSpikeTimes(p, 500)
    # the oracle copies the initial state, so it is built before simulating
    net = cc.oracle_network(ngpu, pops, gens, d, seed=seed)
    ngpu.Simulate(1200.0)
    g_steps, g_nodes = _gpu_spikes(ngpu, first[0], n_total)
    net.simulate(12000)
    o_steps, o_nodes = net.spikes()
    assert len(o_steps) > 1000
    # early spike trains (first 30 ms after the first spike)
    t_first = int(o_steps.min())
    hit, tot = _match_fraction(o_steps, o_nodes, g_steps, g_nodes, t_first + 300)
    assert tot > 0 and hit >= 0.99 * tot, (hit, tot)
    g_rates, g_cv = cc.rates_and_cv(g_steps, g_nodes, first, sizes, 2000, 12000)
    o_rates, o_cv = cc.rates_and_cv(o_steps, o_nodes, first, sizes, 2000, 12000)
    print("rates gpu   ", np.round(g_rates, 3))
    print("rates oracle", np.round(o_rates, 3))
    for k in range(len(pops)):
        counts = o_rates[k] * sizes[k] * 1.0
        tol = 3.0 / np.sqrt(max(counts, 1.0)) + 0.05
        assert abs(g_rates[k] - o_rates[k]) <= tol * o_rates[k] + 1e-9, (k, g_rates, o_rates)
        if len(o_cv[k]) >= 20 and len(g_cv[k]) >= 20:
            p = stats.ks_2samp(g_cv[k], o_cv[k]).pvalue
            print("ISI-CV", cc.POPS[k], len(g_cv[k]), len(o_cv[k]), "KS p", p)
            assert p > 1e-3, (k, p)


def test_cortical_column_full_scale_rates(ngpu):
    """Full cortical column as the reference's microcircuit script runs it
    (77,169 iaf_psc_exp, about 3e8 synapses, Poisson background, 1 s
    pre-simulation + 10 s, python/Potjans_2014_s/sim_params.py:12-14):
    population rates over the 10 s within 3% of the published rates of the
    model (network_params.py:75-76)."""
    pops, gens, d = cc.build(ngpu, n_scaling=1.0, k_scaling=1.0, seed=12349)
    first, sizes = _pop_bounds(pops)
    for p in pops:
        ngpu.ActivateSpikeCount(p)
    ngpu.Simulate(1000.0)
    c0 = [np.asarray(ngpu.GetNeuronIntVarArray(p.i0, p.n, "spike_count")) for p in pops]
    ngpu.Simulate(10000.0)
    c1 = [np.asarray(ngpu.GetNeuronIntVarArray(p.i0, p.n, "spike_count")) for p in pops]
    rates = np.array([(b - a).sum() / len(a) / 10.0 for a, b in zip(c0, c1)])
    dev = rates / cc.FULL_MEAN_RATES - 1.0
    print("full-scale rates", np.round(rates, 3), "published", cc.FULL_MEAN_RATES,
          "relative deviation", np.round(dev, 4), "wall s (10 s)", ngpu.LastSimulateSeconds())
    assert ngpu.NConnections() > 2.9e8
    assert np.all(np.abs(dev) < 0.03), dev


STDP = {"tau_plus": 20.0, "tau_minus": 20.0, "lambda": 0.01, "alpha": 1.0,
        "mu_plus": 0.0, "mu_minus": 0.0, "Wmax": 0.2}


def _stdp_network(ngpu, n, k, w_pg=0.2, rate=15000.0, seed=4321):
    """Plasticity network: aeif_cond_alpha, fixed in-degree k (80% excitatory
    STDP synapses with initial weights uniform in [0.02, 0.1) nS, 20%
    inhibitory static 0.35 nS), integer delays 1-5 ms, Poisson drive."""
    ngpu.SetKernelStatus("rnd_seed", seed)
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", rate)
    nrn = ngpu.Create("aeif_cond_alpha", n, 2)
    ngpu.SetStatus(nrn, {"E_rev": [0.0, -85.0]})
    ngpu.SetNeuronGroupParam(nrn, "rk5_eps", 1e-3)
    sg = ngpu.CreateSynGroup("stdp", STDP)
    ne = int(0.8 * n)
    exc, inh = nrn[0:ne], nrn[ne:n]
    ke, ki = int(0.8 * k) // 5, (k - int(0.8 * k)) // 5
    for dly in (1.0, 2.0, 3.0, 4.0, 5.0):
        ngpu.Connect(exc, nrn, {"rule": "fixed_indegree", "indegree": ke},
                     {"weight": {"distribution": "uniform", "low": 0.02, "high": 0.1},
                      "delay": dly, "receptor": 0, "synapse_group": sg})
        ngpu.Connect(inh, nrn, {"rule": "fixed_indegree", "indegree": ki},
                     {"weight": 0.35, "delay": dly, "receptor": 1})
    ngpu.Connect(pg, nrn, {"rule": "all_to_all"}, {"weight": w_pg, "delay": 0.1, "receptor": 0})
    return pg, nrn, sg


def _stdp_oracle(ngpu, nrn, w_pg, rate, seed):
    from oracle import oracle as orc
    net = orc.Network(dt=0.1, seed=seed)
    net.create(orc.POISSON_GENERATOR, 1, params={"rate": rate})
    net.create(orc.AEIF_COND_ALPHA, nrn.n, 2, params={"E_rev": [0.0, -85.0]}, eps=1e-3)
    net.syn_group("stdp", STDP)
    c = ngpu.GetAllConnections()
    net.connect(c["source"], c["target"], c["port"], c["weight"], c["delay"], c["syn"])
    return net, c


def test_stdp_network_vs_oracle(ngpu):
    """Plasticity network at 2,000 neurons x in-degree 1000 (1.6e6 STDP
    synapses), 500 ms: weights exact while the spike trains agree, then the
    final weight histogram against the oracle."""
    n, k, w_pg, rate, seed = 2000, 1000, 0.2, 15000.0, 4321
    pg, nrn, sg = _stdp_network(ngpu, n, k, w_pg, rate, seed)
    ngpu.ActivateRecSpikeTimes(nrn, 1000)
    net, c0 = _stdp_oracle(ngpu, nrn, w_pg, rate, seed)
    plastic = c0["syn"] == 1
    assert np.count_nonzero(plastic) == n * (int(0.8 * k) // 5) * 5
    # phase 1 (40 ms, the first volleys): a plastic synapse whose source and
    # target emitted identical spike trains on both sides has the same weight
    t_done = 40.0
    ngpu.Simulate(t_done)
    net.simulate(400)
    o_steps, o_nodes = net.spikes()
    g_steps, g_nodes = _gpu_spikes(ngpu, nrn.i0, n)
    ol, gl = {}, {}
    for s_, n_ in sorted(zip(o_steps.tolist(), o_nodes.tolist())):
        ol.setdefault(n_, []).append(s_)
    for s_, n_ in sorted(zip(g_steps.tolist(), g_nodes.tolist())):
        gl.setdefault(n_, []).append(s_)
    agree = np.zeros(nrn.i0 + n, dtype=bool)
    for i in range(nrn.i0, nrn.i0 + n):
        agree[i] = ol.get(i, []) == gl.get(i, [])
    wg = ngpu.GetAllConnections()["weight"]
    wo = net.weights(len(wg))
    both = plastic & agree[c0["source"]] & agree[c0["target"]]
    changed = both & (np.abs(wg - c0["weight"]) > 1e-6)
    print("phase 1: oracle spikes", len(o_steps), "gpu spikes", len(g_steps),
          "neurons agreeing", int(agree.sum()), "synapses compared", int(both.sum()),
          "of which changed", int(changed.sum()))
    assert len(o_steps) > 0 and agree.sum() >= 0.9 * n
    assert changed.sum() > 1000
    assert np.max(np.abs(wg[both] - wo[both])) < 1e-5
    # phase 2: to 500 ms
    ngpu.Simulate(500.0 - t_done)
    net.simulate(int(round((500.0 - t_done) / 0.1)))
    wg = ngpu.GetAllConnections()["weight"][plastic]
    wo = net.weights(len(c0["weight"]))[plastic]
    assert wg.min() >= 0.0 and wg.max() <= STDP["Wmax"] + 1e-6
    bins = np.linspace(0.0, STDP["Wmax"], 21)
    hg = np.histogram(wg, bins)[0] / len(wg)
    ho = np.histogram(wo, bins)[0] / len(wo)
    l1 = float(np.abs(hg - ho).sum())
    print("weight histogram gpu   ", np.round(hg, 4))
    print("weight histogram oracle", np.round(ho, 4))
    print("L1", l1, "mean", wg.mean(), wo.mean(), "w0 mean", c0["weight"][plastic].mean())
    assert np.abs(wg - c0["weight"][plastic]).max() > 1e-3     # plasticity acted
    assert l1 < 0.1
    assert abs(wg.mean() - wo.mean()) < 0.02 * wo.mean()


def test_stdp_network_full_scale(ngpu):
    """Plasticity network at full size (100,000 aeif_cond_alpha x in-degree
    1000, 8e7 STDP synapses), 1 s: weights stay in [0, Wmax], static
    synapses keep their weight, the histogram is printed for the record."""
    n, k = 100000, 1000
    pg, nrn, sg = _stdp_network(ngpu, n, k, 0.2, 15000.0, 99)
    c0 = ngpu.GetAllConnections()
    ngpu.Simulate(1000.0)
    c1 = ngpu.GetAllConnections()
    plastic = c0["syn"] == 1
    w = c1["weight"][plastic]
    assert w.min() >= 0.0 and w.max() <= STDP["Wmax"] + 1e-6
    assert np.array_equal(c1["weight"][~plastic], c0["weight"][~plastic])
    hist = np.histogram(w, np.linspace(0.0, STDP["Wmax"], 21))[0] / len(w)
    print("full-scale STDP: wall s", ngpu.LastSimulateSeconds(), "spikes", ngpu.TotalSpikes(),
          "mean w", w.mean(), "hist", np.round(hist, 4))
    assert ngpu.TotalSpikes() > 0


# step modes: several steps per launch (windows, the default where the
# delays allow), and one step per launch with the delivery in the update's
# grid, on a forked stream, or serial
DELIVERY_ENV = {"window": {}, "fused": {"NGB200_WINDOW": "0"},
                "fork": {"NGB200_WINDOW": "0", "NGB200_FUSE_DELIVERY": "0"},
                "serial": {"NGB200_WINDOW": "0", "NGB200_FUSE_DELIVERY": "0",
                           "NGB200_FORK_DELIVERY": "0"}}


def _chunk_run(ngpu, chunk, mode):
    """mode: one step mode, or one per Simulate call (the mode switches
    between the calls)."""
    import os
    keys = ("NGB200_FUSE_DELIVERY", "NGB200_FORK_DELIVERY", "NGB200_WINDOW")
    modes = [mode] * 3 if isinstance(mode, str) else list(mode)
    old = {k: os.environ.get(k) for k in keys}

    def set_mode(m):
        for k in keys:
            os.environ.pop(k, None)
        os.environ.update(DELIVERY_ENV[m])
    set_mode(modes[0])
    try:
        b = ngpu.default_binding()
        b.Reset()
        b.SetVerbosityLevel(0)
        ngpu.SetKernelStatus("rnd_seed", 99)
        pg = ngpu.Create("poisson_generator")
        ngpu.SetStatus(pg, "rate", 20000.0)
        nrn = ngpu.Create("aeif_cond_beta", 2000, 2)
        ngpu.SetStatus(nrn, {"E_rev": [0.0, -85.0], "tau_rise": [0.2, 0.5],
                             "tau_decay": [2.0, 8.0]})
        ngpu.Connect(pg, nrn, {"rule": "all_to_all"}, {"weight": 0.5, "delay": 0.1,
                                                       "receptor": 0})
        ngpu.Connect(nrn[0:1600], nrn, {"rule": "fixed_indegree", "indegree": 80},
                     {"weight": 0.05, "delay": 1.5, "receptor": 0})
        ngpu.Connect(nrn[1600:2000], nrn, {"rule": "fixed_indegree", "indegree": 20},
                     {"weight": 0.35, "delay": 0.7, "receptor": 1})
        ngpu.ActivateSpikeCount(nrn)
        b.SetGraphChunk(chunk)
        totals = []
        for t, m in zip((33.3, 50.0, 16.7), modes):
            set_mode(m)
            ngpu.Simulate(t)
            totals.append(b.TotalSpikes())
        counts = ngpu.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count")
        v = np.asarray(ngpu.GetNeuronVar(nrn.i0, nrn.n, "V_m"), dtype=np.float32).ravel()
        return totals, counts, v
    finally:
        for k in keys:
            if old[k] is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = old[k]


def test_step_chunks_and_spike_totals(ngpu):
    """Each step of a captured chunk reads its own copy of the step context
    and the delivery does the step bookkeeping: graphs of 100, 7 and 1 steps,
    no graph at all, windows of several steps per launch (5 steps in chunks
    of 100 at the 0.7 ms shortest delay, 7 in chunks of 7), and one step per
    launch with the delivery in the update's grid, on a forked stream or
    serial, and switches between windows and one step per launch between
    Simulate calls, give bit-identical state, and the running spike total
    equals the sum of the per-neuron spike counts after every Simulate
    call."""
    ref = _chunk_run(ngpu, 100, "fused")
    assert ref[1].sum() > 100
    assert ref[0][-1] == int(ref[1].sum())
    assert ref[0][0] < ref[0][1] < ref[0][2]
    for chunk, mode in ((7, "fused"), (1, "fused"), (0, "fused"), (100, "fork"), (7, "fork"),
                        (100, "serial"), (100, "window"), (7, "window"), (1, "window"),
                        (100, ("window", "fused", "window")),
                        (7, ("fork", "window", "serial"))):
        totals, counts, v = _chunk_run(ngpu, chunk, mode)
        assert totals == ref[0], (chunk, mode)
        assert np.array_equal(counts, ref[1]), (chunk, mode)
        assert np.array_equal(v.view(np.int32), ref[2].view(np.int32)), (chunk, mode)


def test_window_spike_totals_with_generator_connections_only(ngpu):
    """Windows of up to 16 steps where no connection goes through the spike
    ring (Poisson generators only: their 0.1 ms delay does not bound the
    window): every step of a window keeps its own ring slot, so the running
    spike total equals the per-neuron counts and the one-step run's."""
    import os
    out = []
    for window in ("16", "0"):
        os.environ["NGB200_WINDOW"] = window
        try:
            b = ngpu.default_binding()
            b.Reset()
            b.SetVerbosityLevel(0)
            ngpu.SetKernelStatus("rnd_seed", 5)
            pg = ngpu.Create("poisson_generator")
            ngpu.SetStatus(pg, "rate", 20000.0)
            nrn = ngpu.Create("aeif_cond_beta", 4096, 2)
            ngpu.SetStatus(nrn, {"I_e": 1000.0})
            ngpu.Connect(pg, nrn, {"rule": "all_to_all"}, {"weight": 0.6, "delay": 0.1,
                                                           "receptor": 0})
            ngpu.ActivateSpikeCount(nrn)
            ngpu.Simulate(20.0)
            counts = ngpu.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count")
            out.append((b.TotalSpikes(), counts, b.KernelsPerStep()))
        finally:
            os.environ.pop("NGB200_WINDOW", None)
    (tw, cw, kw), (ts, cs, ks) = out
    assert kw < 0.5 < ks                        # the first run used windows
    assert cw.sum() > 10000
    assert np.array_equal(cw, cs)
    assert tw == int(cw.sum()) == ts


def _mixed_window_net(ngpu, window):
    import os
    os.environ["NGB200_WINDOW"] = window
    try:
        b = ngpu.default_binding()
        b.Reset()
        b.SetVerbosityLevel(0)
        ngpu.SetKernelStatus("rnd_seed", 2024)
        pg1 = ngpu.Create("poisson_generator")
        ngpu.SetStatus(pg1, "rate", 12000.0)
        pg2 = ngpu.Create("poisson_generator")
        ngpu.SetStatus(pg2, "rate", 30000.0)
        a = ngpu.Create("aeif_cond_alpha", 1000, 2)
        c = ngpu.Create("aeif_cond_beta", 1500, 2)
        ngpu.SetStatus(c, {"E_rev": [0.0, -85.0], "tau_rise": [0.2, 0.5],
                           "tau_decay": [2.0, 8.0]})
        p = ngpu.Create("aeif_psc_exp", 800, 2)
        groups = (a, c, p)
        for g in groups:
            # per-neuron draws from two generators (the per-connection path
            # of the Poisson input, not the uniform drive)
            ngpu.Connect(pg1, g, {"rule": "all_to_all"}, {"weight": 0.4, "delay": 0.1,
                                                          "receptor": 0})
            ngpu.Connect(pg2, g[0:g.n // 2], {"rule": "all_to_all"},
                         {"weight": 0.2, "delay": 0.3, "receptor": 0})
        delay = {"distribution": "uniform", "low": 1.0, "high": 2.0}
        for src in groups:
            for tgt in groups:
                ngpu.Connect(src, tgt, {"rule": "fixed_indegree", "indegree": 30},
                             {"weight": 0.05 if tgt is not p else 5.0, "delay": delay,
                              "receptor": 0})
        ngpu.Connect(p[0:200], c, {"rule": "fixed_indegree", "indegree": 10},
                     {"weight": 0.3, "delay": 1.4, "receptor": 1})
        for g in groups:
            ngpu.ActivateRecSpikeTimes(g, 200)
        ngpu.Simulate(40.0)
        ngpu.Simulate(23.7)
        kps = b.KernelsPerStep()
        out = []
        for g in groups:
            v = np.asarray(ngpu.GetNeuronVar(g.i0, g.n, "V_m"), dtype=np.float32).view(np.int32)
            times = [np.asarray(ngpu.GetRecSpikeTimes(g[i]), dtype=np.float32)
                     for i in range(0, g.n, 7)]
            out.append((v, times))
        return out, b.TotalSpikes(), kps
    finally:
        os.environ.pop("NGB200_WINDOW", None)


def test_windows_mixed_models_per_connection_poisson(ngpu):
    """Windows (10 steps at the 1.0 ms shortest delay) against one step per
    launch on three RK5 models with per-neuron Poisson inputs from two
    generators, a uniformly distributed delay and recorded spike times:
    every membrane potential, every recorded spike time and the spike total
    agree bit for bit."""
    w, tw, kw = _mixed_window_net(ngpu, "16")
    s, ts, ks = _mixed_window_net(ngpu, "0")
    assert kw < 0.6 < ks
    assert ts == tw and ts > 1000
    for (vw, timew), (vs, times) in zip(w, s):
        assert np.array_equal(vw, vs)
        for a, b in zip(timew, times):
            assert np.array_equal(a, b)


def _busy_net(ngpu, env):
    """40,000 aeif_cond_beta at about 25 Hz with in-degree 1000: about 1e5
    delivered events per step, a busy network (the event rate is checked
    after every chunk of the first 1000 steps)."""
    import os
    keys = ("NGB200_WINDOW", "NGB200_BUSY_MODE")
    old = {k: os.environ.get(k) for k in keys}
    for k in keys:
        os.environ.pop(k, None)
    os.environ.update(env)
    try:
        b = ngpu.default_binding()
        b.Reset()
        b.SetVerbosityLevel(0)
        ngpu.SetKernelStatus("rnd_seed", 17)
        n = 40000
        pg = ngpu.Create("poisson_generator")
        ngpu.SetStatus(pg, "rate", 20000.0)
        nrn = ngpu.Create("aeif_cond_beta", n, 2)
        ngpu.SetStatus(nrn, {"E_rev": [0.0, -85.0], "tau_rise": [1.0, 1.0],
                             "tau_decay": [1.0, 1.0]})
        ngpu.Connect(pg, nrn, {"rule": "all_to_all"}, {"weight": 0.5, "delay": 0.1,
                                                       "receptor": 0})
        ngpu.Connect(nrn[0:32000], nrn, {"rule": "fixed_indegree", "indegree": 800},
                     {"weight": 0.05, "delay": 1.0, "receptor": 0})
        ngpu.Connect(nrn[32000:n], nrn, {"rule": "fixed_indegree", "indegree": 200},
                     {"weight": 0.35, "delay": 1.5, "receptor": 1})
        ngpu.ActivateSpikeCount(nrn)
        ngpu.Simulate(150.0)
        ev0 = b.DeliveredEvents()
        ngpu.Simulate(50.0)
        ev_step = (b.DeliveredEvents() - ev0) / 500.0
        counts = ngpu.GetNeuronIntVarArray(nrn.i0, nrn.n, "spike_count")
        v = np.asarray(ngpu.GetNeuronVar(nrn.i0, nrn.n, "V_m"), dtype=np.float32).ravel()
        return v, counts, b.TotalSpikes(), b.KernelsPerStep(), ev_step
    finally:
        for k in keys:
            if old[k] is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = old[k]


def test_busy_network_windows_match_one_step_per_launch(ngpu):
    """A busy network in windows (its lanes going through a window's steps
    each at its own pace, the delivery before each window) against one step
    per launch: every membrane potential, every spike count and the spike
    total agree bit for bit."""
    vw, cw, tw, kw, ew = _busy_net(ngpu, {"NGB200_BUSY_MODE": "2"})
    vs, cs, ts, ks, es = _busy_net(ngpu, {"NGB200_WINDOW": "0"})
    assert ew > 65536 and es == ew          # busy, the same events
    assert kw < 0.5 < ks                    # the first run used windows
    assert tw == ts == int(cw.sum())
    assert np.array_equal(cw, cs)
    assert np.array_equal(vw.view(np.int32), vs.view(np.int32))
