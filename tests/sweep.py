"""Parameter sweep of independent AdEx networks (the batched workload): each
network is its own aeif_cond_beta node group with its own Poisson generator,
recurrent fixed in-degree connections inside the network only, and its own
adaptation parameters a, b and input rate drawn on a seeded grid."""
import numpy as np

NEURON = {"E_rev": [0.0, -85.0], "tau_rise": [0.2, 0.5], "tau_decay": [2.0, 8.0]}


def sweep_grid(n_nets, n_min, n_max, k_min, k_max, seed=2024):
    """Sizes log-uniform in [n_min, n_max], in-degrees uniform in
    [k_min, k_max], a in [0, 8] nS, b in [0, 150] pA, rate in [10, 30] kHz."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_nets)).astype(int)
    k = rng.integers(k_min, k_max + 1, n_nets)
    a = rng.uniform(0.0, 8.0, n_nets)
    b = rng.uniform(0.0, 150.0, n_nets)
    rate = rng.uniform(10000.0, 30000.0, n_nets)
    return [dict(n=int(sizes[i]), k=int(k[i]), a=float(a[i]), b=float(b[i]),
                 rate=float(rate[i])) for i in range(n_nets)]


def build_sweep(ngpu, grid, w_pg=0.2, w_exc=0.05, w_inh=0.35, eps=1e-3, seed=1234):
    """Creates every network of the grid through the API; returns the
    neuron groups. Integer delays 1 and 2 ms, half of the inputs each."""
    ngpu.SetKernelStatus("rnd_seed", seed)
    nets = []
    for p in grid:
        pg = ngpu.Create("poisson_generator")
        ngpu.SetStatus(pg, "rate", p["rate"])
        nrn = ngpu.Create("aeif_cond_beta", p["n"], 2)
        par = dict(NEURON)
        par["a"] = p["a"]
        par["b"] = p["b"]
        ngpu.SetStatus(nrn, par)
        ngpu.SetNeuronGroupParam(nrn, "rk5_eps", eps)
        ne = int(0.8 * p["n"])
        ke = max(1, int(0.8 * p["k"]) // 2)
        ki = max(1, (p["k"] - int(0.8 * p["k"])) // 2)
        for d in (1.0, 2.0):
            ngpu.Connect(nrn[0:ne], nrn, {"rule": "fixed_indegree", "indegree": ke},
                         {"weight": w_exc, "delay": d, "receptor": 0})
            ngpu.Connect(nrn[ne:p["n"]], nrn, {"rule": "fixed_indegree", "indegree": ki},
                         {"weight": w_inh, "delay": d, "receptor": 1})
        ngpu.Connect(pg, nrn, {"rule": "all_to_all"}, {"weight": w_pg, "delay": 0.1, "receptor": 0})
        nets.append(nrn)
    return nets
