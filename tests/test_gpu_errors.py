"""Device error paths, made to fire without a fault or a hang (needs a B200).

Every failure here is produced by a host setting: a spike list that is too
small, an RK5 sub-step limit of 2, or the wait-test hook that makes a
bounded device wait give up after one non-blocking test (the kernel then
still waits, bounded, for its own copies and tensor-core work before it
exits). Each test checks that Simulate reports the mapped error (the
reference's code 2, a ValueError in Python) and that the process and its
device context keep working afterwards.

The reference reports these conditions with printf and exit
(src/send_spike.cu:37-41, src/spike_buffer.cu:188-209); it has no
counterpart of the wait time-outs.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _still_works(ngpu):
    """A fresh small network runs and gives the expected single-neuron
    trace after the error (the context is usable)."""
    from tests import netdefs
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    t, v = netdefs.run_single_api(ngpu, "aeif_cond_beta")
    assert netdefs.nest_rmse(v, "aeif_cond_beta") <= 5e-4


def test_spike_ring_overflow_is_reported(ngpu):
    n = 200
    sg = ngpu.Create("spike_generator")
    ngpu.SetStatus(sg, {"spike_times": [1.0], "spike_heights": [1.0]})
    par = ngpu.Create("parrot_neuron", n)
    ngpu.Connect(sg, par, {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0})
    # capacity ceil(201 * 0.001) = 1 spike per step: the parrots' volley overflows
    ngpu.SetKernelStatus("max_spike_num_fact", 0.001)
    with pytest.raises(ValueError, match="more spikes in one step"):
        ngpu.Simulate(5.0)
    assert ngpu.GetErrorCode() == 2
    _still_works(ngpu)


def test_rk5_substep_limit_is_reported(ngpu):
    # the first steps start from the initial step size (1e-2 dt) and need
    # several sub-steps: a limit of 2 trips
    nrn = ngpu.Create("aeif_cond_beta", 64, 2)
    ngpu.SetRk5MaxSubsteps(2)
    with pytest.raises(ValueError, match="substep limit"):
        ngpu.Simulate(1.0)
    ngpu.SetRk5MaxSubsteps(200000)
    ngpu.Simulate(1.0)                 # the limit back: no error
    v = ngpu.GetNeuronVar(nrn.i0, nrn.n, "V_m")
    assert np.all(np.isfinite(np.asarray(v, dtype=np.float64)))
    _still_works(ngpu)


def test_tile_prefetch_timeout_is_reported(ngpu, monkeypatch):
    # the persistent variant with shared-memory prefetch (uniform parameters),
    # a kernel of one step per launch
    monkeypatch.setenv("NGB200_RK5_VARIANT", "7")
    monkeypatch.setenv("NGB200_WINDOW", "0")
    nrn = ngpu.Create("aeif_cond_beta", 20000, 2)
    ngpu.Simulate(0.5)
    assert ngpu.GetRk5Tuning(nrn.i0)[0] == 7
    ngpu.SetWaitTest(1)
    with pytest.raises(ValueError, match="prefetch of the RK5 update timed out"):
        ngpu.Simulate(0.5)
    msg = ngpu.GetErrorMessage()
    assert "device state lost" not in msg      # the copies in flight drained
    ngpu.SetWaitTest(0)
    ngpu.Simulate(0.5)                          # normal waits again: no error
    _still_works(ngpu)


def _proposer_net(ngpu):
    from oracle import mlp
    rng = np.random.default_rng(3)
    P = rng.normal(0.0, 0.3, mlp.NPARAM).astype(np.float32)
    P[mlp.B3] = -2.0
    ngpu.SetKernelStatus("rnd_seed", 5)
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", 20000.0)
    nrn = ngpu.Create("aeif_cond_beta", 4096, 2)
    ngpu.SetNeuronGroupParam(nrn, "rk5_eps", 1e-3)
    # a strong constant current: the neurons spike from the first
    # milliseconds, so steps of several sub-steps (the proposer's) occur
    ngpu.SetStatus(nrn, {"I_e": 1000.0})
    ngpu.Connect(pg, nrn, {"rule": "all_to_all"}, {"weight": 0.6, "delay": 0.1, "receptor": 0})
    ngpu.SetStepProposerParams(P)
    ngpu.SetStepProposer(nrn, True)
    return nrn


@pytest.mark.parametrize("mask", [1, 2])
def test_proposer_wait_timeout_is_reported(ngpu, mask):
    """mask 1: the first tensor-core wait of a proposal round gives up;
    mask 2: the second one (layer 2 still in flight when the round fails,
    so the teardown must wait for that completion before it frees the
    tensor memory). The CTA falls back to the plain controller. The
    proposer runs for neurons that need more than one sub-step in a step
    (the straggler queue's records): 20 ms lets the driven neurons reach
    their first spikes."""
    nrn = _proposer_net(ngpu)
    ngpu.SetWaitTest(mask)
    with pytest.raises(ValueError, match="step proposer timed out"):
        ngpu.Simulate(20.0)
    ngpu.SetWaitTest(0)
    ngpu.Simulate(2.0)
    v = np.asarray(ngpu.GetNeuronVar(nrn.i0, nrn.n, "V_m"), dtype=np.float64)
    assert np.all(np.isfinite(v))
    _still_works(ngpu)
