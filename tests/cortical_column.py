"""Layered cortical-column network (Potjans & Diesmann 2014) built through the
NeuronGPU Python API, as the reference's microcircuit example builds it
(python/Potjans_2014_s/network.py:240-330 with the parameters of
python/Potjans_2014_s/network_params.py:29-130 and sim_params.py:12-20).

The model parameters below are the published values shipped with the
reference; the derived quantities (synapse numbers, PSC amplitudes, in-degree
scaling compensation) are computed here from their defining formulas.
"""
import numpy as np

POPS = ["L23E", "L23I", "L4E", "L4I", "L5E", "L5I", "L6E", "L6I"]
FULL_NUM_NEURONS = np.array([20683, 5834, 21915, 5479, 4850, 1065, 14395, 2948])
# population rates (spikes/s) of the full-scale model (network_params.py:75-76)
FULL_MEAN_RATES = np.array([0.943, 3.026, 4.368, 5.882, 7.733, 8.664, 1.096, 7.851])
# connection probability target <- source (network_params.py:79-88)
CONN_PROBS = np.array(
    [[0.1009, 0.1689, 0.0437, 0.0818, 0.0323, 0., 0.0076, 0.],
     [0.1346, 0.1371, 0.0316, 0.0515, 0.0755, 0., 0.0042, 0.],
     [0.0077, 0.0059, 0.0497, 0.135, 0.0067, 0.0003, 0.0453, 0.],
     [0.0691, 0.0029, 0.0794, 0.1597, 0.0033, 0., 0.1057, 0.],
     [0.1004, 0.0622, 0.0505, 0.0057, 0.0831, 0.3726, 0.0204, 0.],
     [0.0548, 0.0269, 0.0257, 0.0022, 0.06, 0.3158, 0.0086, 0.],
     [0.0156, 0.0066, 0.0211, 0.0166, 0.0572, 0.0197, 0.0396, 0.2252],
     [0.0364, 0.001, 0.0034, 0.0005, 0.0277, 0.008, 0.0658, 0.1443]])
K_EXT = np.array([1600, 1500, 2100, 1900, 2000, 1900, 2900, 2100])
BG_RATE = 8.0
PSP_EXC = 0.15
G_REL = -4.0
WEIGHT_REL_STD = 0.1
DELAY_EXC, DELAY_INH, DELAY_REL_STD = 1.5, 0.75, 0.5
DELAY_POISSON = 1.5
V0_MEAN = [-68.28, -63.16, -63.33, -63.45, -63.11, -61.66, -66.72, -61.43]
V0_STD = [5.36, 4.57, 4.74, 4.94, 4.94, 4.55, 5.46, 4.48]
NEURON = {"E_L": -65.0, "V_th": -50.0, "V_reset": -65.0, "C_m": 250.0, "tau_m": 10.0,
          "tau_syn": 0.5, "t_ref": 2.0}


def psc_over_psp(C_m, tau_m, tau_syn):
    """PSC amplitude (pA) per mV of PSP peak for an exponential current into a
    leaky membrane: v(t) = J a (e^{-t/tau_m} - e^{-t/tau_syn}) / C_m with
    a = tau_m tau_syn / (tau_m - tau_syn), maximal at
    t* = a ln(tau_m / tau_syn)."""
    a = tau_m * tau_syn / (tau_m - tau_syn)
    t_peak = a * np.log(tau_m / tau_syn)
    psp_per_pa = a / C_m * (np.exp(-t_peak / tau_m) - np.exp(-t_peak / tau_syn))
    return 1.0 / psp_per_pa


def num_synapses(conn_probs, n_post, n_pre):
    """Total synapse number K for which K draws with replacement over all
    n_post x n_pre pairs hit a given pair with probability conn_probs."""
    prod = np.outer(n_post, n_pre).astype(float)
    return np.log(1.0 - conn_probs) / np.log((prod - 1.0) / prod)


def derive(n_scaling=1.0, k_scaling=1.0):
    """Neuron and synapse numbers, weights and compensating DC input of the
    scaled model (network.py:130-200; in-degree scaling compensation as in the
    microcircuit model: weights / sqrt(k), mean input restored by DC)."""
    npop = len(POPS)
    full_syn = num_synapses(CONN_PROBS, FULL_NUM_NEURONS, FULL_NUM_NEURONS)
    n = np.round(FULL_NUM_NEURONS * n_scaling).astype(int)
    syn = np.round(full_syn * n_scaling * k_scaling).astype(int)
    k_ext = np.round(K_EXT * k_scaling).astype(int)
    fac = psc_over_psp(NEURON["C_m"], NEURON["tau_m"], NEURON["tau_syn"])
    psp = np.zeros((npop, npop))
    psp[:, 0::2] = PSP_EXC
    psp[:, 1::2] = PSP_EXC * G_REL
    psp[0, 2] = 2.0 * PSP_EXC
    w = psp * fac
    w_ext = PSP_EXC * fac
    dc = np.zeros(npop)
    if k_scaling != 1.0:
        sk = np.sqrt(k_scaling)
        indeg = full_syn / FULL_NUM_NEURONS[:, None]
        input_rec = np.sum(w * indeg * FULL_MEAN_RATES, axis=1)
        dc = dc + 0.001 * NEURON["tau_syn"] * (1.0 - sk) * input_rec
        dc = dc + 0.001 * NEURON["tau_syn"] * (1.0 - sk) * w_ext * K_EXT * BG_RATE
        w = w / sk
        w_ext = w_ext / sk
    return {"n": n, "syn": syn, "k_ext": k_ext, "w": w, "w_ext": w_ext, "dc": dc}


def build(ngpu, n_scaling=1.0, k_scaling=1.0, seed=12349, dt=0.1):
    """Creates the populations, Poisson background and recurrent synapses
    through the API; returns (populations, generators, derived numbers)."""
    d = derive(n_scaling, k_scaling)
    ngpu.SetRandomSeed(seed)
    pops = []
    E_L = NEURON["E_L"]
    for i in range(len(POPS)):
        p = ngpu.Create("iaf_psc_exp", int(d["n"][i]))
        ngpu.SetStatus(p, {"tau_ex": NEURON["tau_syn"], "tau_in": NEURON["tau_syn"],
                           "E_L": E_L, "Theta_rel": NEURON["V_th"] - E_L,
                           "V_reset_rel": NEURON["V_reset"] - E_L,
                           "t_ref": NEURON["t_ref"], "I_e": float(d["dc"][i])})
        ngpu.SetStatus(p, {"V_m_rel": {"distribution": "normal", "mu": V0_MEAN[i] - E_L,
                                       "sigma": V0_STD[i]}})
        pops.append(p)
    gens = ngpu.Create("poisson_generator", len(POPS))
    for i in range(len(POPS)):
        ngpu.SetStatus([gens[i]], "rate", float(BG_RATE * d["k_ext"][i]))
    for i, tgt in enumerate(pops):
        for j, src in enumerate(pops):
            if d["syn"][i][j] <= 0:
                continue
            w_mean = float(d["w"][i][j])
            w_std = abs(w_mean * WEIGHT_REL_STD)
            if w_mean < 0:
                w_lo, w_hi, rec = w_mean - 3.0 * w_std, 0.0, 1
            else:
                w_lo, w_hi, rec = 0.0, w_mean + 3.0 * w_std, 0
            d_mean = DELAY_EXC if j % 2 == 0 else DELAY_INH
            d_std = d_mean * DELAY_REL_STD
            ngpu.Connect(src, tgt, {"rule": "fixed_total_number", "total_num": int(d["syn"][i][j])},
                         {"weight": {"distribution": "normal_clipped", "mu": w_mean,
                                     "low": w_lo, "high": w_hi, "sigma": w_std},
                          "delay": {"distribution": "normal_clipped", "mu": d_mean,
                                    "low": dt, "high": d_mean + 3.0 * d_std, "sigma": d_std},
                          "receptor": rec})
    for i, tgt in enumerate(pops):
        ngpu.Connect([gens[i]], tgt, {"rule": "all_to_all"},
                     {"weight": float(d["w_ext"]), "delay": DELAY_POISSON})
    return pops, gens, d


def oracle_network(ngpu, pops, gens, d, seed, dt=0.1):
    """The same network on the FP64 oracle: identical nodes, initial
    membrane potentials, parameters and every connection (read back in bulk),
    so that the Poisson draws agree draw by draw. Call it before the first
    simulation: it copies the current membrane potentials."""
    from oracle import oracle as orc
    net = orc.Network(dt=dt, seed=seed)
    E_L = NEURON["E_L"]
    for i, p in enumerate(pops):
        v0 = np.asarray(ngpu.GetStatus(p, "V_m_rel"), dtype=np.float64).reshape(-1)
        net.create(orc.IAF_PSC_EXP, len(v0), 2,
                   params={"tau_ex": NEURON["tau_syn"], "tau_in": NEURON["tau_syn"],
                           "E_L": E_L, "Theta_rel": NEURON["V_th"] - E_L,
                           "V_reset_rel": NEURON["V_reset"] - E_L,
                           "t_ref": NEURON["t_ref"], "I_e": float(np.float32(d["dc"][i]))},
                   vars={"V_m_rel": v0})
    rates = np.array([float(np.float32(BG_RATE * d["k_ext"][i])) for i in range(len(pops))])
    net.create(orc.POISSON_GENERATOR, len(pops), 0, params={"rate": rates})
    c = ngpu.GetAllConnections()
    net.connect(c["source"], c["target"], c["port"], c["weight"], c["delay"], c["syn"])
    return net


def rates_and_cv(spike_steps, spike_nodes, pops_first, pops_n, t0_step, t1_step, dt=0.1):
    """Per-population mean rate (spikes/s) in steps [t0, t1) and per-neuron
    ISI coefficients of variation (neurons with >= 3 spikes)."""
    m = (spike_steps >= t0_step) & (spike_steps < t1_step)
    st, nd = spike_steps[m], spike_nodes[m]
    dur = (t1_step - t0_step) * dt * 1e-3
    rates, cvs = [], []
    order = np.lexsort((st, nd))
    st, nd = st[order], nd[order]
    for first, n in zip(pops_first, pops_n):
        sel = (nd >= first) & (nd < first + n)
        rates.append(np.count_nonzero(sel) / n / dur)
        s2, n2 = st[sel], nd[sel]
        cv = []
        bounds = np.searchsorted(n2, np.arange(first, first + n + 1))
        for k in range(n):
            t = s2[bounds[k]:bounds[k + 1]]
            if len(t) >= 3:
                isi = np.diff(t).astype(float)
                cv.append(isi.std() / isi.mean())
        cvs.append(np.asarray(cv))
    return np.asarray(rates), cvs
