"""Learned RK5 step proposer: training kernels, tensor-core inference and the
gain over the plain controller. Needs a B200.

Tolerances:
  * training gradients (FP32 kernels) against the FP64 oracle: within 1e-4 of
    the largest gradient component;
  * tensor-core inference against the oracle's emulation of its BF16 inputs
    and FP32 accumulation: 2e-3 + 2e-3 |output|; against the FP64 network:
    0.15 (BF16 rounding of inputs and weights);
  * learned vs plain controller on the same neurons: every step still passes
    the same RK5 error test, so the spike trains agree within one step for
    >= 99% of spikes and the spike count within 1%.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand_params(rng, scale=0.4):
    from oracle import mlp
    P = rng.normal(0.0, scale, mlp.NPARAM).astype(np.float32)
    P[mlp.B3] = -2.0
    return P


def test_training_gradients_match_oracle(ngpu):
    from oracle import mlp
    rng = np.random.default_rng(1)
    P = _rand_params(rng)
    data = np.zeros((3000, 8), dtype=np.float32)
    data[:, :6] = rng.normal(0.0, 1.0, (3000, 6))
    data[:, 6] = rng.normal(-3.0, 1.5, 3000)
    g, loss = ngpu.MlpGradients(data, P)
    lo, go = mlp.loss_and_grad(P.astype(np.float64), data.astype(np.float64))
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    scale = np.max(np.abs(go))
    assert np.max(np.abs(g - go)) <= 1e-4 * scale, np.max(np.abs(g - go)) / scale


def test_tensor_core_inference_matches_oracle(ngpu):
    from oracle import mlp
    rng = np.random.default_rng(2)
    P = _rand_params(rng, 0.3)
    X = rng.normal(0.0, 1.0, (1000, 6)).astype(np.float32)     # 7 full CTAs + a partial one
    out = ngpu.MlpInfer(X, P)
    ref_tc = mlp.forward_tensor_core(P, X)
    ref64, _ = mlp.forward(P.astype(np.float64), X.astype(np.float64))
    err_tc = np.abs(out - ref_tc)
    print("tensor-core inference: max |gpu - bf16 oracle|", err_tc.max(),
          "max |gpu - fp64 oracle|", np.max(np.abs(out - ref64)))
    assert np.all(err_tc <= 2e-3 + 2e-3 * np.abs(ref_tc)), err_tc.max()
    assert np.max(np.abs(out - ref64)) < 0.15


def _driven_neurons(ngpu, n, w_pg, rate=20000.0, seed=77):
    """n unconnected aeif_cond_beta neurons (config[0] parameters, b = 0),
    each with its own Poisson input: the spike trains of two integrators can
    be compared neuron by neuron without network chaos."""
    ngpu.SetKernelStatus("rnd_seed", seed)
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", rate)
    nrn = ngpu.Create("aeif_cond_beta", n, 2)
    ngpu.SetStatus(nrn, {"E_rev": [0.0, -85.0], "tau_rise": [0.2, 0.5], "tau_decay": [2.0, 8.0],
                         "b": 0.0, "a": 1.0})
    ngpu.SetNeuronGroupParam(nrn, "rk5_eps", 1e-3)
    ngpu.Connect(pg, nrn, {"rule": "all_to_all"}, {"weight": w_pg, "delay": 0.1, "receptor": 0})
    ngpu.ActivateRecSpikeTimes(nrn, 2000)
    return nrn


def _spikes(ngpu, nrn):
    out = []
    for i in range(nrn.n):
        out.append(np.rint(np.asarray(ngpu.GetRecSpikeTimes(nrn[i])) / 0.1).astype(np.int64))
    return out


def test_learned_proposer_gain(ngpu):
    """Log accepted sub-steps of the plain controller, train on the GPU,
    then run the same neurons with the plain and the learned controller:
    fewer stage evaluations, same spikes within one step."""
    n, w_pg, t_log, t_run = 8192, 0.6, 300.0, 500.0
    nrn = _driven_neurons(ngpu, n, w_pg)
    ngpu.SetStepLog(nrn, 1 << 20)
    ngpu.Simulate(t_log)
    logged = ngpu.GetStepLogCount(nrn)
    rows, l0, l1 = ngpu.TrainStepProposer(steps=3000, blocks=64, lr=3e-3, seed=11)
    params = ngpu.GetStepProposerParams()
    print("logged", logged, "trained rows", rows, "loss first", l0, "last", l1)
    assert rows > 10000 and l1 < 0.5 * l0

    runs = {}
    for mode in ("plain", "learned"):
        ngpu.Reset()
        nrn = _driven_neurons(ngpu, n, w_pg)
        if mode == "learned":
            ngpu.SetStepProposerParams(params)
            ngpu.SetStepProposer(nrn, True)
        ngpu.Simulate(t_run)
        runs[mode] = (ngpu.StageEvaluations(), _spikes(ngpu, nrn), ngpu.LastSimulateDeviceMs())
    e0, s0, ms0 = runs["plain"]
    e1, s1, ms1 = runs["learned"]
    n0 = sum(len(s) for s in s0)
    n1 = sum(len(s) for s in s1)
    matched = 0
    for a, b in zip(s0, s1):
        for t in a:
            if len(b) and np.min(np.abs(b - t)) <= 1:
                matched += 1
    steps = n * t_run / 0.1
    print("stage evaluations per neuron-step plain %.4f learned %.4f (reduction %.1f%%)"
          % (e0 / steps, e1 / steps, 100.0 * (1.0 - e1 / e0)))
    print("spikes plain", n0, "learned", n1, "rate %.2f Hz" % (n0 / n / (t_run * 1e-3)),
          "matched within one step %.4f" % (matched / max(n0, 1)),
          "device ms plain %.1f learned %.1f" % (ms0, ms1))
    assert n0 > 0
    assert e1 < e0
    assert matched >= 0.99 * n0
    assert abs(n1 - n0) <= 0.01 * n0
