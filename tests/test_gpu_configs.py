"""Parity on the configurations the benchmark runs, and the reference's own
network-rate test (needs a B200).

* The small configuration exactly as the benchmark states it (1000
  aeif_cond_beta, 800 exc / 200 inh, fixed in-degree 100 with w 0.05 / 0.35
  nS, integer delays 1-2 ms, Poisson 20 kHz w 0.05 nS, RK5 tolerance 1e-3,
  seed 1234, 1 s), built by bench.build_network, against the FP64 oracle
  loaded with the connections the GPU built: membrane traces to 1e-4 of the
  70 mV scale while both are silent, rates if anything fires.
* The scale configuration (1e6 neurons x 1000 synapses, tolerance 1e-3):
  every 1000th neuron recorded for 100 ms. While the network stays silent
  (checked) every neuron sees only its own Poisson drive, so the sample is
  replayed exactly by the oracle with the same random streams.
* python/test/test_brunel_list.py of the reference: 1000 aeif_cond_beta,
  fixed in-degree CE = 800 / CI = 200 (every source once), normal_clipped
  delays, Poisson 20 kHz w 0.37, 1 s; out- and in-degree checks and its
  acceptance: every recorded neuron within 30.78 +- 3 sqrt(30.78) spikes,
  the mean of the 100 within 3 sqrt(30.78) / sqrt(100).
"""
import math

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


def _oracle_params():
    return {k: (np.float32(v) if np.isscalar(v) else [np.float32(x) for x in v])
            for k, v in bench.NEURON_PARAMS.items()}


def test_config_small_vs_oracle(ngpu):
    from oracle import oracle as orc
    cfg = dict(bench.SMALL)
    b = ngpu.default_binding()
    pg, nrn = bench.build_network(ngpu, cfg, seed=1234)
    sample = list(range(0, cfg["n"], 10))
    rec = ngpu.CreateRecord("", ["V_m"] * len(sample), [nrn[i] for i in sample], [0] * len(sample))
    ngpu.ActivateRecSpikeTimes(nrn, 100)
    n_steps = 10000
    ngpu.Simulate(n_steps * 0.1)
    gv = np.asarray(ngpu.GetRecordData(rec))[1:, 1:]
    g_spikes = b.TotalSpikes()
    net = orc.Network(dt=0.1, seed=1234)
    net.create(orc.POISSON_GENERATOR, 1, params={"rate": cfg["rate"]})
    net.create(orc.AEIF_COND_BETA, cfg["n"], 2, params=_oracle_params(), eps=cfg["eps"])
    c = ngpu.GetAllConnections()
    assert len(c["source"]) == cfg["n"] * (cfg["k_exc"] + cfg["k_inh"]) + cfg["n"]
    net.connect(c["source"], c["target"], c["port"], c["weight"], c["delay"], c["syn"])
    ov = net.simulate(n_steps, record=[(nrn[i], 0) for i in sample])
    o_steps, _ = net.spikes()
    first = int(o_steps.min()) if len(o_steps) else n_steps
    err = float(np.max(np.abs(gv[:first] - ov[:first]))) / 70.0
    print("small configuration: gpu spikes %d, oracle spikes %d, max |dV| / 70 mV before the "
          "first spike %.3g over %d steps" % (g_spikes, len(o_steps), err, first))
    assert first > 100
    assert err < 1e-4, err
    if len(o_steps) or g_spikes:
        # rates over the whole second, within 3 sigma + 5 % of the oracle's
        r_o, r_g = len(o_steps) / cfg["n"], g_spikes / cfg["n"]
        assert abs(r_g - r_o) <= 3.0 * math.sqrt(max(r_o, 1.0) / cfg["n"]) + 0.05 * r_o


def test_config_scale_sample_vs_oracle(ngpu):
    from oracle import oracle as orc
    cfg = dict(bench.SCALE)
    b = ngpu.default_binding()
    pg, nrn = bench.build_network(ngpu, cfg, seed=1234)
    sample = np.arange(0, cfg["n"], 1000)
    rec = ngpu.CreateRecord("", ["V_m"] * len(sample), [nrn[int(i)] for i in sample],
                            [0] * len(sample))
    n_steps = 1000
    ngpu.Simulate(n_steps * 0.1)
    gv = np.asarray(ngpu.GetRecordData(rec))[1:, 1:]
    # silent: no neuron received recurrent input, each saw only its own drive
    assert b.TotalSpikes() == 0
    net = orc.Network(dt=0.1, seed=1234)
    net.create(orc.POISSON_GENERATOR, 1, params={"rate": cfg["rate"]})
    net.create(orc.AEIF_COND_BETA, len(sample), 2, params=_oracle_params(), eps=cfg["eps"])
    net.connect(np.zeros(len(sample), dtype=np.int32), np.arange(len(sample)) + 1, 0,
                cfg["w_pg"], 0.1)
    # the drive of neuron i uses random stream i (one generator, all_to_all in order)
    net.set_direct_streams(sample.astype(np.uint64))
    ov = net.simulate(n_steps, record=[(1 + k, 0) for k in range(len(sample))])
    err = float(np.max(np.abs(gv - ov))) / 70.0
    swing = float(np.max(ov) - np.min(ov))
    print("scale configuration sample: %d neurons, %d steps, V range %.3f mV, max |dV| / 70 mV "
          "%.3g" % (len(sample), n_steps, swing, err))
    assert swing > 0.5             # the drive moved the membranes
    assert err < 1e-4, err


def test_reference_brunel_rate(ngpu):
    order, n_test, expected_rate = 200, 100, 30.78
    NE, NI = 4 * order, order
    n = NE + NI
    CE, CI = 800, 200
    rng = np.random.default_rng(1234)
    ngpu.SetKernelStatus("rnd_seed", 1234)
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", 20000.0)
    neuron = ngpu.Create("aeif_cond_beta", n, 2)
    exc, inh = neuron[0:NE], neuron[NE:n]
    ngpu.SetStatus(neuron, {"E_rev": [0.0, -85.0], "tau_decay": [1.0, 1.0],
                            "tau_rise": [1.0, 1.0]})
    delay = {"distribution": "normal_clipped", "mu": 0.5, "low": 0.1, "high": 0.5 + 3 * 0.25,
             "sigma": 0.25}
    ngpu.Connect(exc, neuron.ToList(), {"rule": "fixed_indegree", "indegree": CE},
                 {"weight": 0.05, "delay": delay, "receptor": 0})
    ngpu.Connect(inh.ToList(), exc.ToList(), {"rule": "fixed_indegree", "indegree": CI},
                 {"weight": 0.35, "delay": delay, "receptor": 1})
    ngpu.Connect(inh.ToList(), inh, {"rule": "fixed_indegree", "indegree": CI},
                 {"weight": 0.35, "delay": delay, "receptor": 1})
    ngpu.Connect(pg.ToList(), neuron.ToList(), {"rule": "all_to_all"},
                 {"weight": 0.37, "delay": 0.2, "receptor": 0})
    rec_nodes = [neuron[0], neuron[n - 1]] + [neuron[int(i)] for i in rng.integers(0, n, n_test - 2)]
    rec = ngpu.CreateRecord("", ["spike"] * n_test, rec_nodes, [0] * n_test)
    ngpu.Simulate()
    data = np.asarray(ngpu.GetRecordData(rec))
    for i in range(n):
        assert len(ngpu.GetConnections(i + 1)) == NE + NI, i
    for i in rng.integers(0, n, 10):
        assert len(ngpu.GetConnections(target=int(i) + 1)) == NE + NI + 1, i
    spikes = data[:, 1:].sum(axis=0)
    lo = expected_rate - 3.0 * math.sqrt(expected_rate)
    hi = expected_rate + 3.0 * math.sqrt(expected_rate)
    mean = float(spikes.mean())
    print("Brunel network: mean rate %.2f Hz (expected %.2f +- %.2f), min %d, max %d"
          % (mean, expected_rate, 3.0 * math.sqrt(expected_rate) / math.sqrt(n_test),
             spikes.min(), spikes.max()))
    assert spikes.min() >= lo and spikes.max() <= hi
    assert abs(mean - expected_rate) <= 3.0 * math.sqrt(expected_rate) / math.sqrt(n_test)
