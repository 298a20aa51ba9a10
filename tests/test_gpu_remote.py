"""A network partitioned over two hosts against the same network on one
(needs a B200).

The reference runs a network over several hosts with RemoteCreate /
RemoteConnect and an MPI exchange of the spikes every step
(python/test/test_brunel_mpi.py, src/neurongpu.cu:490-521). Here the two
hosts are two simulator instances in one process on one GPU, and the
exchange that the Python layer runs with torch.distributed between
processes is done by hand between them: after each run of E steps (the
shortest remote delay) each host packs the spikes of its exported nodes,
and each unpacks the other's list into its image nodes. A third instance
holds the whole network with ordinary connections. Deterministic drive
(a different constant current per neuron slice) and deterministic rules
make the two runs comparable spike for spike: every spike time, the final
membrane potentials bit for bit, and the spike totals (image nodes are not
counted) must agree.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 100                     # neurons per host
T_MS = 300.0
# (weight, delay ms, port) per connection; A on host 0, B on host 1
AA = (0.02, 1.2, 0)         # all_to_all
BB = (0.2, 0.8, 1)          # all_to_all
AB = (0.05, 1.0, 0)         # all_to_all, remote from host 0 to host 1
BA = (0.5, 1.5, 1)          # one_to_one, remote from host 1 to host 0
I_E = [600.0 + 60.0 * k for k in range(10)]     # pA, per slice of 10 neurons


def _population(ngpu):
    nrn = ngpu.Create("aeif_cond_beta", N, 2)
    ngpu.SetStatus(nrn, {"E_rev": [0.0, -85.0], "tau_rise": [0.2, 0.5],
                         "tau_decay": [2.0, 8.0]})
    for k, ie in enumerate(I_E):
        ngpu.SetStatus(nrn[10 * k:10 * (k + 1)], {"I_e": ie})
    ngpu.ActivateRecSpikeTimes(nrn, 1000)
    return nrn


def _syn(c):
    return {"weight": c[0], "delay": c[1], "receptor": c[2]}


def _spike_times(ngpu, nrn):
    return [np.asarray(ngpu.GetRecSpikeTimes(nrn[i]), dtype=np.float32) for i in range(nrn.n)]


def _state(ngpu, nrn):
    return np.asarray(ngpu.GetNeuronVar(nrn.i0, nrn.n, "V_m"), dtype=np.float32).view(np.int32)


def test_partitioned_network_matches_single_host(ngpu):
    import torch
    b = ngpu.default_binding()
    A = ngpu.NodeSeq(0, N)
    B = ngpu.NodeSeq(0, N)
    try:
        # the whole network on one host
        b.SetInstance(1)
        b.Reset()
        b.SetVerbosityLevel(0)
        a1 = _population(ngpu)
        b1 = _population(ngpu)
        ngpu.Connect(a1, a1, {"rule": "all_to_all"}, _syn(AA))
        ngpu.Connect(b1, b1, {"rule": "all_to_all"}, _syn(BB))
        ngpu.Connect(a1, b1, {"rule": "all_to_all"}, _syn(AB))
        ngpu.Connect(b1, a1, {"rule": "one_to_one"}, _syn(BA))
        ngpu.Simulate(T_MS)
        ref_a, ref_b = _spike_times(ngpu, a1), _spike_times(ngpu, b1)
        ref_va, ref_vb = _state(ngpu, a1), _state(ngpu, b1)
        ref_total = b.TotalSpikes()
        # the same network on two hosts: A on host 0, B on host 1; every
        # host makes the same calls, as the scripts of a partitioned run do
        pops = {}
        for inst, host in ((2, 0), (3, 1)):
            b.SetInstance(inst)
            b.Reset()
            b.SetVerbosityLevel(0)
            b.SetHost(host, 2)
            pops[host] = _population(ngpu)
            own = pops[host]
            syn_local = AA if host == 0 else BB
            ngpu.Connect(own, own, {"rule": "all_to_all"}, _syn(syn_local))
            ngpu.RemoteConnect(0, own if host == 0 else A, 1, own if host == 1 else B,
                               {"rule": "all_to_all"}, _syn(AB))
            ngpu.RemoteConnect(1, own if host == 1 else B, 0, own if host == 0 else A,
                               {"rule": "one_to_one"}, _syn(BA))
        e_steps = []
        for inst in (2, 3):
            b.SetInstance(inst)
            b.SetSimTime(T_MS)
            b.StartSimulation()
            e_steps.append(b.RemoteExchangeSteps())
        # host 1 receives over 1.0 ms, host 0 over 1.5 ms (and exports)
        assert e_steps[1] == 10 and e_steps[0] == 15
        E = min(e_steps)
        cap = N * E                      # at most one spike per node and step
        bufs = [torch.zeros(4 + 3 * cap, dtype=torch.int32, device="cuda") for _ in range(2)]
        n_steps = int(round(T_MS / 0.1))
        exchanged = 0
        for _ in range(n_steps // E):
            counts = []
            for inst, host in ((2, 0), (3, 1)):
                b.SetInstance(inst)
                b.SimulateSteps(E)
                counts.append(b.PackRemoteSpikes(E, bufs[host].data_ptr(), cap))
            assert max(counts) <= cap
            b.SetInstance(2)
            b.UnpackRemoteSpikes(1, E, bufs[1].data_ptr(), counts[1])
            b.SetInstance(3)
            b.UnpackRemoteSpikes(0, E, bufs[0].data_ptr(), counts[0])
            torch.cuda.synchronize()
            exchanged += sum(counts)
        totals = []
        for inst, host in ((2, 0), (3, 1)):
            b.SetInstance(inst)
            b.EndSimulation()
            totals.append(b.TotalSpikes())
        b.SetInstance(2)
        got_a, got_va = _spike_times(ngpu, pops[0]), _state(ngpu, pops[0])
        b.SetInstance(3)
        got_b, got_vb = _spike_times(ngpu, pops[1]), _state(ngpu, pops[1])
        n_ref = sum(len(s) for s in ref_a) + sum(len(s) for s in ref_b)
        print("spikes", n_ref, "exchanged", exchanged, "totals", totals, ref_total)
        assert n_ref > 500 and exchanged > 200
        for g, r in zip(got_a + got_b, ref_a + ref_b):
            assert np.array_equal(g, r)
        assert np.array_equal(got_va, ref_va) and np.array_equal(got_vb, ref_vb)
        assert totals[0] + totals[1] == ref_total
    finally:
        for inst in (3, 2, 1):
            b.SetInstance(inst)
            b.Reset()
        b.SetInstance(0)


def _brunel_host(ngpu, b, host):
    """One host of the reference's two-host Brunel test
    (python/test/test_brunel_mpi.py): 400 excitatory and 100 inhibitory
    aeif_cond_beta per host, local and remote connections with fixed
    in-degrees, normal-clipped delays, a Poisson drive of 20 kHz at 0.37 nS."""
    b.Reset()
    b.SetVerbosityLevel(0)
    b.SetHost(host, 2)
    ngpu.SetKernelStatus("rnd_seed", 1234)
    NE, NI, CE, CI = 400, 100, 800, 200
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", 20000.0)
    neuron = ngpu.Create("aeif_cond_beta", NE + NI, 2)
    exc, inh = neuron[0:NE], neuron[NE:NE + NI]
    ngpu.SetStatus(neuron, {"E_rev": [0.0, -85.0], "tau_decay": [1.0, 1.0],
                            "tau_rise": [1.0, 1.0]})
    delay = {"distribution": "normal_clipped", "mu": 0.5, "low": 0.1, "high": 0.5 + 3 * 0.25,
             "sigma": 0.25}
    exc_syn = {"weight": 0.05, "delay": delay, "receptor": 0}
    inh_syn = {"weight": 0.35, "delay": delay, "receptor": 1}
    ngpu.Connect(exc, neuron, {"rule": "fixed_indegree", "indegree": CE // 2}, exc_syn)
    ngpu.Connect(inh, exc, {"rule": "fixed_indegree", "indegree": CI // 2}, inh_syn)
    ngpu.Connect(inh, inh, {"rule": "fixed_indegree", "indegree": CI // 2}, inh_syn)
    ngpu.Connect(pg, neuron, {"rule": "all_to_all"},
                 {"weight": 0.37, "delay": 0.2, "receptor": 0})
    for src_host, tgt_host in ((0, 1), (1, 0)):
        ngpu.RemoteConnect(src_host, exc, tgt_host, neuron,
                           {"rule": "fixed_indegree", "indegree": CE // 2}, exc_syn)
    for src_host, tgt_host in ((0, 1), (1, 0)):
        ngpu.RemoteConnect(src_host, inh, tgt_host, neuron,
                           {"rule": "fixed_indegree", "indegree": CI // 2}, inh_syn)
    ngpu.ActivateSpikeCount(neuron)
    return neuron


def test_reference_two_host_brunel(ngpu):
    """The reference's two-host test on two instances: every local neuron
    connects to all NE + NI local neurons, every neuron receives
    2 (NE + NI) + 1 connections (the remote ones from image nodes), and the
    spike count of 100 sampled neurons per host over 1 s lies within the
    reference's acceptance, 30.78 +- 3 sqrt(30.78)
    (python/test/test_brunel_mpi.py:11,135-175). The exchange runs every step
    (the shortest remote delay is 0.1 ms)."""
    import math
    import torch
    b = ngpu.default_binding()
    NE, NI = 400, 100
    try:
        nrn = {}
        for inst, host in ((4, 0), (5, 1)):
            b.SetInstance(inst)
            nrn[host] = _brunel_host(ngpu, b, host)
        e_steps = []
        for inst in (4, 5):
            b.SetInstance(inst)
            b.SetSimTime(1000.0)
            b.StartSimulation()
            e_steps.append(b.RemoteExchangeSteps())
            for i in range(NE + NI):
                assert len(ngpu.GetConnections(i + 1)) == NE + NI
            for i in (1, 137, 250, 412, 500):
                assert len(ngpu.GetConnections(target=i)) == 2 * (NE + NI) + 1
        E = min(e_steps)
        assert E == 1
        cap = (NE + NI) * E
        bufs = [torch.zeros(4 + 3 * cap, dtype=torch.int32, device="cuda") for _ in range(2)]
        for _ in range(10000 // E):
            counts = []
            for inst, host in ((4, 0), (5, 1)):
                b.SetInstance(inst)
                b.SimulateSteps(E)
                counts.append(b.PackRemoteSpikes(E, bufs[host].data_ptr(), cap))
            b.SetInstance(4)
            b.UnpackRemoteSpikes(1, E, bufs[1].data_ptr(), counts[1])
            b.SetInstance(5)
            b.UnpackRemoteSpikes(0, E, bufs[0].data_ptr(), counts[0])
            torch.cuda.synchronize()
        rng = np.random.default_rng(7)
        expected = 30.78
        lo, hi = expected - 3.0 * math.sqrt(expected), expected + 3.0 * math.sqrt(expected)
        for inst, host in ((4, 0), (5, 1)):
            b.SetInstance(inst)
            b.EndSimulation()
            counts = ngpu.GetNeuronIntVarArray(nrn[host].i0, nrn[host].n, "spike_count")
            sample = [0, NE + NI - 1] + list(rng.integers(0, NE + NI, 98))
            s = counts[sample]
            print("host", host, "mean rate %.2f Hz" % counts.mean(), "sample min", s.min(),
                  "max", s.max())
            assert lo <= s.min() and s.max() <= hi
    finally:
        for inst in (5, 4):
            b.SetInstance(inst)
            b.Reset()
        b.SetInstance(0)
