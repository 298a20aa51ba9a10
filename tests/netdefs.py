"""Shared definitions of the test networks, built both through the drop-in
API (CUDA core) and on the FP64 oracle.

The single-neuron cases restate the reference's own test scripts
(python/test/test_aeif_cond_beta.py:5-40, test_aeif_cond_alpha.py,
test_aeif_psc_alpha.py, test_aeif_psc_exp.py, test_aeif_psc_delta.py,
test_iaf_psc_exp.py, test_iaf_psc_exp_g.py, test_iaf_psc_exp_hc.py,
test_izh.py): one neuron driven by a spike generator firing at 10 and 400 ms
(10 and 40 ms for izhikevich) through one connection per receptor port, V_m
recorded every step for 800 ms (80 ms) and compared with NEST at 1 ms
resolution.
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

SINGLE = {
    "aeif_cond_beta": dict(
        n_port=3, var="V_m", tol=5e-4,
        params={"V_peak": 0.0, "a": 4.0, "b": 80.5, "E_L": -70.6, "g_L": 300.0,
                "E_rev": [20.0, 0.0, -85.0], "tau_decay": [40.0, 20.0, 30.0],
                "tau_rise": [20.0, 10.0, 5.0]},
        conns=[(0, 0.1, 1.0), (1, 0.2, 100.0), (2, 0.5, 130.0)]),
    "aeif_cond_alpha": dict(
        n_port=3, var="V_m", tol=5e-4,
        params={"V_peak": 0.0, "a": 4.0, "b": 80.5, "E_L": -70.6, "g_L": 300.0,
                "E_rev": [20.0, 0.0, -85.0], "tau_syn": [40.0, 20.0, 30.0]},
        conns=[(0, 0.1, 1.0), (1, 0.2, 100.0), (2, 0.5, 130.0)]),
    "aeif_psc_alpha": dict(
        n_port=2, var="V_m", tol=5e-4,
        params={"V_peak": 0.0, "a": 4.0, "b": 80.5, "E_L": -70.6, "g_L": 300.0,
                "tau_syn": [40.0, 20.0]},
        conns=[(0, 1.0, 1.0), (1, -2.0, 100.0)]),
    "aeif_psc_exp": dict(
        n_port=2, var="V_m", tol=5e-4,
        params={"V_peak": 0.0, "a": 4.0, "b": 80.5, "E_L": -70.6, "g_L": 300.0,
                "tau_syn": [40.0, 20.0]},
        conns=[(0, 1.0, 1.0), (1, -2.0, 100.0)]),
    "aeif_psc_delta": dict(
        n_port=1, var="V_m", tol=5e-4,
        params={"V_peak": 0.0, "a": 4.0, "b": 80.5, "E_L": -70.6, "g_L": 300.0,
                "C_m": 20000.0},
        conns=[(0, 1.0, 1.0), (0, -2.0, 100.0)]),
    "iaf_psc_exp": dict(
        n_port=2, var="V_m_rel", tol=5e-5, params={}, offset=-70.0,
        conns=[(0, 1.0, 1.0), (1, -2.0, 100.0)]),
    # python/test/test_iaf_psc_exp_g.py, test_iaf_psc_exp_hc.py: both
    # connections on the single port, E_L = -65 mV, NEST trace
    # test_fast_iaf_psc_exp_nest.txt, tolerance 5e-4
    "iaf_psc_exp_g": dict(
        n_port=1, var="V_m_rel", tol=5e-4, params={}, offset=-65.0,
        golden="fast_iaf_psc_exp", conns=[(0, 1.0, 1.0), (0, -2.0, 100.0)]),
    "iaf_psc_exp_hc": dict(
        n_port=1, var="V_m_rel", tol=5e-4, params={}, offset=-65.0,
        golden="fast_iaf_psc_exp", conns=[(0, 1.0, 1.0), (0, -2.0, 100.0)],
        oracle="iaf_psc_exp_g", oracle_params={"h_prop": 0.1}),
    # python/test/test_izh.py: spikes at 10 and 40 ms, delays 1 and 10 ms,
    # 80 ms, NEST trace test_izh_nest.txt, tolerance 5e-3
    "izhikevich": dict(
        n_port=1, var="V_m", tol=5e-3, params={}, golden="izh",
        spikes=[10.0, 40.0], sim=80.0, conns=[(0, 1.0, 1.0), (0, -2.0, 10.0)]),
}
# user_m1: the reference's user-model template, shipped as a copy of
# aeif_cond_beta (src/user_m1_kernel.h)
SINGLE["user_m1"] = dict(SINGLE["aeif_cond_beta"], golden="aeif_cond_beta",
                         oracle="aeif_cond_beta")
SPIKE_TIMES = [10.0, 400.0]
SIM_TIME = 800.0


def n_samples(name):
    """recorded rows of a single-neuron case: initial state plus one per step"""
    return int(round(SINGLE[name].get("sim", SIM_TIME) / 0.1)) + 1


def golden(name):
    fname = SINGLE[name].get("golden", name) if name in SINGLE else name
    return np.loadtxt(os.path.join(GOLDEN, "nest_%s.txt" % fname), delimiter="\t")


def nest_rmse(v_m, name):
    """The reference's acceptance metric: std(dV)/|mean(V)| with the
    simulated trace sampled at rows i*10+20 against NEST row i."""
    g = golden(name)
    # test_iaf_psc_exp.py:29 records V_m_rel and adds E_L = -70 mV
    v = np.asarray(v_m) + SINGLE[name].get("offset", 0.0)
    dv = [v[i * 10 + 20] - g[i, 1] for i in range(len(g))]
    return float(np.std(dv) / abs(np.mean(v)))


def run_single_api(ngpu, name):
    c = SINGLE[name]
    neuron = ngpu.Create(name, 1, c["n_port"])
    if c["params"]:
        ngpu.SetStatus(neuron, c["params"])
    sg = ngpu.Create("spike_generator")
    ngpu.SetStatus(sg, {"spike_times": c.get("spikes", SPIKE_TIMES)})
    for port, w, d in c["conns"]:
        syn = {"weight": w, "delay": d}
        if c["n_port"] > 1:
            syn["receptor"] = port
        ngpu.Connect(sg, neuron, {"rule": "all_to_all"}, syn)
    rec = ngpu.CreateRecord("", [c["var"]], [neuron[0]], [0])
    ngpu.Simulate(c.get("sim", SIM_TIME))
    data = np.asarray(ngpu.GetRecordData(rec))
    return data[:, 0], data[:, 1]


def _oracle_models():
    from oracle import oracle as orc
    return {"aeif_cond_beta": orc.AEIF_COND_BETA, "aeif_cond_alpha": orc.AEIF_COND_ALPHA,
            "aeif_psc_alpha": orc.AEIF_PSC_ALPHA, "aeif_psc_exp": orc.AEIF_PSC_EXP,
            "aeif_psc_delta": orc.AEIF_PSC_DELTA, "iaf_psc_exp": orc.IAF_PSC_EXP,
            "iaf_psc_exp_g": orc.IAF_PSC_EXP_G, "izhikevich": orc.IZHIKEVICH,
            "izhikevich_psc_exp": orc.IZH_PSC_EXP, "izhikevich_cond_beta": orc.IZH_COND_BETA}


class _LazyModels(dict):
    def __missing__(self, key):
        self.update(_oracle_models())
        return dict.__getitem__(self, key)


ORACLE_MODEL = _LazyModels()


def run_single_oracle(name, eps=1e-6):
    from oracle import oracle as orc
    c = SINGLE[name]
    model = ORACLE_MODEL[c.get("oracle", name)]
    net = orc.Network(dt=0.1)
    params = {k: (np.float32(v) if np.isscalar(v) else [np.float32(x) for x in v])
              for k, v in dict(c["params"], **c.get("oracle_params", {})).items()}
    neuron = net.create(model, 1, c["n_port"], params=params, eps=eps)
    sg = net.create(orc.SPIKE_GENERATOR, 1)
    net.set_spikes(sg, [c.get("spikes", SPIKE_TIMES)])
    for port, w, d in c["conns"]:
        net.connect([sg.i0], [neuron.i0], port, w, d)
    n_steps = int(round(c.get("sim", SIM_TIME) / 0.1))
    vi = neuron.var_index(c["var"])
    tr = net.simulate(n_steps, record=[(neuron.i0, vi)])[:, 0]
    v0 = net_initial(model, c)
    t = np.arange(n_steps + 1) * np.float32(0.1)
    return t, np.concatenate([[v0], tr]), net


def net_initial(model, c):
    from oracle import oracle as orc
    sv, svd = orc.MODELS[model][0], orc.MODELS[model][1]
    return svd[sv.index(c["var"])] if c["var"] not in c["params"] else c["params"][c["var"]]
