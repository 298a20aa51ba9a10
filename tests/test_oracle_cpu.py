"""The FP64 oracle pinned against the reference's golden vectors (CPU only).

Pins: the NEST membrane traces shipped with the reference (single-neuron
tests, acceptance metric of python/test/test_aeif_cond_beta.py:46-50), the
closed-form STDP expectation of python/test/test_stdp.py:5-18, the published
Philox4x32-10 known-answer vectors, and the Poisson sampler's moments.
"""
import math

import numpy as np
import pytest

from tests import netdefs
from oracle import oracle as orc


@pytest.mark.parametrize("name", sorted(netdefs.SINGLE))
def test_oracle_matches_nest_golden_trace(name):
    t, v, _ = netdefs.run_single_oracle(name)
    assert len(v) == netdefs.n_samples(name)
    rmse = netdefs.nest_rmse(v, name)
    assert rmse <= netdefs.SINGLE[name]["tol"], (name, rmse)


def _stdp_expect(w, Dt, tau_plus, tau_minus, Wplus, alpha, mu_plus, mu_minus, Wmax):
    # python/test/test_stdp.py:5-18
    if Dt >= 0:
        w1 = w + Wplus * math.exp(-Dt / tau_plus) * math.pow(1.0 - w / Wmax, mu_plus)
        return min(w1, Wmax)
    w1 = w - alpha * Wplus * math.exp(Dt / tau_minus) * math.pow(w / Wmax, mu_minus)
    return max(w1, 0.0)


def stdp_pair_network(net_builder_n=50, dt_step=5.0):
    """Pairs of neurons forced to spike once each with a controlled time
    difference (python/test/test_stdp.py:20-70)."""
    N = net_builder_n
    dts = [dt_step * (-0.5 * (N - 1) + i) for i in range(N)]
    return N, dts


@pytest.mark.parametrize("den_delay", [0.0, 3.0])
def test_oracle_stdp_closed_form(den_delay):
    """With a dendritic delay d of the post-synaptic neurons their spikes
    reach the synapses d later: the pair difference becomes Dt + d."""
    N, dts = stdp_pair_network()
    tau_plus = tau_minus = 20.0
    Wmax = 0.001
    net = orc.Network(dt=0.1)
    sg = net.create(orc.SPIKE_GENERATOR, N)
    n0 = net.create(orc.AEIF_COND_BETA, N, 1, params={"t_ref": 1000.0})
    n1 = net.create(orc.AEIF_COND_BETA, N, 1, params={"t_ref": 1000.0, "den_delay": den_delay})
    net.set_spikes(sg, [[50.0]] * N)
    syn = net.syn_group("stdp", {"tau_plus": tau_plus, "tau_minus": tau_minus, "lambda": 1.0,
                                 "alpha": 1.0, "mu_plus": 1.0, "mu_minus": 1.0, "Wmax": Wmax})
    net.connect(np.arange(N) + sg.i0, np.arange(N) + n0.i0, 0, 17.9, 1.0)
    net.connect(np.arange(N) + sg.i0, np.arange(N) + n1.i0, 0, 17.9, 401.0)
    delays = [400.0 - d for d in dts]
    net.connect(np.arange(N) + n0.i0, np.arange(N) + n1.i0, 0, Wmax / 2, delays, syn=syn)
    net.simulate(10000)
    w = net.weights(3 * N)[2 * N:]
    for i in range(N):
        e = _stdp_expect(Wmax / 2, dts[i] + den_delay, tau_plus, tau_minus, 1.0 * Wmax, 1.0, 1.0,
                         1.0, Wmax)
        assert abs(e - w[i]) < 1e-5, (i, dts[i], e, w[i])


def test_philox_known_answers():
    import ctypes
    lib = orc.lib()
    # the oracle links the shared counter-based generator; check it through
    # the Poisson stream of a single draw vs. the published Philox vectors
    # by building the same arithmetic in numpy-free integer Python
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85

    def philox(c, k):
        c = list(c)
        k0, k1 = k
        for _ in range(10):
            p0 = M0 * c[0]
            p1 = M1 * c[2]
            hi0, lo0 = p0 >> 32, p0 & 0xffffffff
            hi1, lo1 = p1 >> 32, p1 & 0xffffffff
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
            k0 = (k0 + W0) & 0xffffffff
            k1 = (k1 + W1) & 0xffffffff
        return c
    assert philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e,
                                                          0xa20bc7c6, 0x6d5451fd]
    assert philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                  [0xa4093822, 0x299f31d0]) == [0xd16cfe09, 0x94fdcceb, 0x5001e420,
                                                0x24126ea1]
    assert lib is not None


def test_oracle_poisson_drive_statistics():
    # 2000 parrot neurons each driven by its own Poisson connection at
    # lambda = rate*dt = 2: per-step counts must be Poisson(2)
    net = orc.Network(dt=0.1, seed=1234)
    pg = net.create(orc.POISSON_GENERATOR, 1, params={"rate": 20000.0})
    par = net.create(orc.PARROT, 2000, 2, params={"hold_spike_height": 1.0})
    net.connect(np.full(2000, pg.i0), np.arange(2000) + par.i0, 0, 1.0, 0.1)
    rec = [(par.i0 + i, 2) for i in range(2000)]
    out = net.simulate(201, record=rec)[1:]   # V = input count of previous step
    counts = out.ravel()
    assert abs(counts.mean() - 2.0) < 0.02
    assert abs(counts.var() - 2.0) < 0.05
    # frequencies of 0..6 against the Poisson pmf
    for k in range(7):
        p = math.exp(-2.0) * 2.0 ** k / math.factorial(k)
        f = np.mean(counts == k)
        assert abs(f - p) < 4 * math.sqrt(p * (1 - p) / counts.size) + 1e-4


def test_mlp_oracle_gradient_finite_differences():
    """The FP64 proposer-network oracle's backpropagation agrees with central
    finite differences (pins the oracle used to check the GPU kernels)."""
    from oracle import mlp
    rng = np.random.default_rng(5)
    P = rng.normal(0.0, 0.3, mlp.NPARAM)
    data = np.concatenate([rng.normal(0.0, 1.0, (50, 6)), rng.normal(-2.0, 1.0, (50, 1))], axis=1)
    loss, g = mlp.loss_and_grad(P, data)
    eps = 1e-6
    for k in list(range(0, mlp.NPARAM, 37)) + [mlp.B3, mlp.W3 + 3, mlp.B1 + 5]:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += eps
        Pm[k] -= eps
        fd = (mlp.loss_and_grad(Pp, data)[0] - mlp.loss_and_grad(Pm, data)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_mlp_oracle_bf16_rounding():
    from oracle import mlp
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-3], dtype=np.float32)
    r = mlp.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0           # tie rounds to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    assert abs(r[4] - 1e-3) < 1e-5


def test_oracle_thread_count_independent():
    """The oracle's parallel node updates give identical results for any
    number of host threads (spikes merged in node order)."""
    def run(threads):
        orc.set_threads(threads)
        rng = np.random.default_rng(3)
        n = 300
        net = orc.Network(dt=0.1, seed=9)
        net.create(orc.POISSON_GENERATOR, 1, params={"rate": 20000.0})
        net.create(orc.AEIF_COND_BETA, n, 2, params={"E_rev": [0.0, -85.0]}, eps=1e-3)
        src = rng.integers(1, n + 1, 20 * n)
        tgt = np.repeat(np.arange(1, n + 1), 20)
        net.connect(src, tgt, 0, 0.5, 1.0)
        net.connect(np.zeros(n, dtype=np.int32), np.arange(1, n + 1), 0, 0.5, 0.1)
        out = net.simulate(300, record=[(5, 0), (77, 0)])
        s, nd = net.spikes()
        return out, s, nd, net.stage_evals()
    a = run(1)
    b = run(4)
    orc.set_threads(1)
    assert len(a[1]) > 0
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2]) and a[3] == b[3]
