"""ctypes wrapper of the FP64 CPU oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
bench.py to check the CUDA core; the product never imports it.

Models and their per-neuron variable / parameter layouts follow the
reference (golosio/NeuronGPU src/*_kernel.h enums); the defaults below are the
reference's NodeInit values (e.g. src/aeif_cond_beta.cu:25-56).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "libngpu_oracle.so")

AEIF_COND_BETA, AEIF_COND_ALPHA, AEIF_PSC_ALPHA, AEIF_PSC_EXP, AEIF_PSC_DELTA, \
    IZH_COND_BETA, IAF_PSC_EXP, SPIKE_GENERATOR, PARROT, POISSON_GENERATOR, \
    IAF_PSC_EXP_G, IZHIKEVICH, IZH_PSC_EXP = range(13)

_AEIF_SCAL = ["V_th", "Delta_T", "g_L", "E_L", "C_m", "a", "b", "tau_w", "I_e",
              "V_peak", "V_reset", "t_ref", "refractory_step", "den_delay"]
_AEIF_DEF = [-50.4, 2.0, 30.0, -70.6, 281.0, 4.0, 80.5, 144.0, 0.0, 0.0, -60.0,
             0.0, 0.0, 0.0]

# name -> (scal vars, scal var defaults, port vars, port var defaults,
#          scal params, defaults, port params, defaults)
MODELS = {
    AEIF_COND_BETA: (["V_m", "w"], [-70.6, 0.0], ["g", "g1"], [0.0, 0.0],
                     _AEIF_SCAL, _AEIF_DEF, ["E_rev", "tau_rise", "tau_decay", "g0"],
                     [0.0, 2.0, 20.0, 0.0]),
    AEIF_COND_ALPHA: (["V_m", "w"], [-70.6, 0.0], ["g", "g1"], [0.0, 0.0],
                      _AEIF_SCAL, _AEIF_DEF, ["E_rev", "tau_syn", "g0"], [0.0, 2.0, 0.0]),
    AEIF_PSC_ALPHA: (["V_m", "w"], [-70.6, 0.0], ["I_syn", "I1_syn"], [0.0, 0.0],
                     _AEIF_SCAL, _AEIF_DEF, ["tau_syn", "I0"], [0.2, 0.0]),
    AEIF_PSC_EXP: (["V_m", "w"], [-70.6, 0.0], ["I_syn"], [0.0],
                   _AEIF_SCAL, _AEIF_DEF, ["tau_syn"], [0.2]),
    AEIF_PSC_DELTA: (["V_m", "w"], [-70.6, 0.0], [], [], _AEIF_SCAL, _AEIF_DEF, [], []),
    IZH_COND_BETA: (["V_m", "u"], [-70.0, -14.0], ["g", "g1"], [0.0, 0.0],
                    ["V_th", "a", "b", "c", "d", "I_e", "t_ref", "refractory_step",
                     "den_delay"], [30.0, 0.02, 0.2, -65.0, 8.0, 0.0, 0.0, 0.0, 0.0],
                    ["E_rev", "tau_rise", "tau_decay", "g0"], [0.0, 2.0, 20.0, 0.0]),
    IAF_PSC_EXP: (["I_syn_ex", "I_syn_in", "V_m_rel", "refractory_step"], [0.0] * 4, [], [],
                  ["tau_m", "C_m", "E_L", "I_e", "Theta_rel", "V_reset_rel", "tau_ex",
                   "tau_in", "t_ref", "den_delay", "P20", "P11ex", "P11in", "P21ex",
                   "P21in", "P22"],
                  [10.0, 250.0, -70.0, 0.0, 15.0, 0.0, 2.0, 2.0, 2.0, 0.0] + [0.0] * 6,
                  [], []),
    SPIKE_GENERATOR: ([], [], [], [], [], [], [], []),
    PARROT: (["input_spike_height", "dummy_input", "V"], [0.0] * 3, [], [],
             ["hold_spike_height", "den_delay"], [0.0, 0.0], [], []),
    POISSON_GENERATOR: ([], [], [], [], ["rate", "origin", "start", "stop"],
                        [0.0, 0.0, 0.0, 1.0e30], [], []),
    # group parameters of the library are per-neuron parameters here;
    # h_prop = 0.1 reproduces iaf_psc_exp_hc (constants fixed at dt 0.1 ms)
    IAF_PSC_EXP_G: (["I_syn", "V_m_rel", "refractory_step"], [0.0] * 3, [], [],
                    ["I_e", "tau_m", "C_m", "E_L", "Theta_rel", "V_reset_rel", "tau_syn",
                     "t_ref", "h_prop"],
                    [0.0, 10.0, 250.0, -65.0, 15.0, 0.0, 0.5, 2.0, 0.0], [], []),
    IZHIKEVICH: (["I_syn", "V_m", "u", "refractory_step"], [0.0, -70.0, -14.0, 0.0], [], [],
                 ["I_e", "den_delay", "V_th", "a", "b", "c", "d", "t_ref"],
                 [0.0, 0.0, 30.0, 0.02, 0.2, -65.0, 8.0, 0.0], [], []),
    IZH_PSC_EXP: (["I_syn", "V_m", "u", "refractory_step"], [0.0, -70.0, -14.0, 0.0], [], [],
                  ["I_e", "den_delay", "V_th", "a", "b", "c", "d", "tau_syn", "t_ref", "n_sub"],
                  [0.0, 0.0, 30.0, 0.02, 0.2, -65.0, 8.0, 0.5, 0.0, 1.0], [], []),
}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)
_llp = ctypes.POINTER(ctypes.c_longlong)


def _load():
    if not os.path.exists(LIB):
        import importlib.util
        spec = importlib.util.spec_from_file_location(
            "build_oracle", os.path.join(HERE, "build_oracle.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = ctypes.CDLL(LIB)
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = (ctypes.c_double, ctypes.c_ulonglong)
    lib.orc_free.argtypes = (ctypes.c_void_p,)
    lib.orc_add_group.restype = ctypes.c_int
    lib.orc_add_group.argtypes = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double)
    lib.orc_set_spikes.argtypes = (ctypes.c_void_p, ctypes.c_int, _ip, _ip, _dp)
    lib.orc_add_syn_group.restype = ctypes.c_int
    lib.orc_add_syn_group.argtypes = (ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int)
    lib.orc_connect.argtypes = (ctypes.c_void_p, ctypes.c_longlong, _ip, _ip, _ip, _ip, _fp, _fp)
    lib.orc_simulate.argtypes = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip, _ip, _dp)
    lib.orc_flush.argtypes = (ctypes.c_void_p,)
    lib.orc_n_spikes.restype = ctypes.c_longlong
    lib.orc_n_spikes.argtypes = (ctypes.c_void_p,)
    lib.orc_get_spikes.argtypes = (ctypes.c_void_p, _llp, _ip)
    lib.orc_get_weights.argtypes = (ctypes.c_void_p, _fp)
    lib.orc_get_state.argtypes = (ctypes.c_void_p, ctypes.c_int, _dp, _dp)
    lib.orc_stage_evals.restype = ctypes.c_longlong
    lib.orc_stage_evals.argtypes = (ctypes.c_void_p,)
    lib.orc_set_threads.argtypes = (ctypes.c_int,)
    lib.orc_rule_edges.restype = ctypes.c_longlong
    lib.orc_rule_edges.argtypes = (ctypes.c_int, ctypes.c_ulonglong, ctypes.c_ulonglong,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip)
    lib.orc_get_threads.restype = ctypes.c_int
    lib.orc_set_direct_streams.argtypes = (ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p)
    lib.orc_set_step_search.argtypes = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int)
    lib.orc_group_evals.restype = ctypes.c_longlong
    lib.orc_group_evals.argtypes = (ctypes.c_void_p, ctypes.c_int)
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def set_threads(n):
    """Host threads of the oracle's parallel node-update loops (results are
    independent of the thread count)."""
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


RULES = {"one_to_one": 0, "all_to_all": 1, "fixed_total_number": 2, "fixed_indegree": 3,
         "fixed_outdegree": 4}


def rule_edges(rule, seed, call, n_source, n_target, param=0):
    """Source and target list indices of a connection rule's connections in
    insertion order (param: total number, in-degree or out-degree)."""
    r = RULES[rule]
    cap = {0: n_source, 1: n_source * n_target}.get(r, 0)
    if r == 2:
        cap = param
    elif r == 3:
        cap = n_target * param
    elif r == 4:
        cap = n_source * param
    s = np.zeros(max(cap, 1), dtype=np.int32)
    t = np.zeros(max(cap, 1), dtype=np.int32)
    m = lib().orc_rule_edges(r, seed, call, n_source, n_target, param, _ptr(s, _ip), _ptr(t, _ip))
    return s[:m], t[:m]


def _ptr(a, t):
    return a.ctypes.data_as(t)


class Group(object):
    def __init__(self, net, model, n, n_port, i0, gid):
        self.net, self.model, self.n, self.n_port, self.i0, self.gid = net, model, n, n_port, i0, gid
        sv, _, pv, _, sp, _, pp, _ = MODELS[model]
        self.var_names = sv + [v + "_%d" % q for q in range(n_port) for v in pv]
        self.param_names = sp + [p + "_%d" % q for q in range(n_port) for p in pp]

    def var_index(self, name, port=0):
        sv, _, pv, _, _, _, _, _ = MODELS[self.model]
        if name in sv:
            return sv.index(name)
        return len(sv) + port * len(pv) + pv.index(name)


class Network(object):
    """A network on the FP64 oracle, built from explicit arrays."""

    def __init__(self, dt=0.1, seed=54321):
        self.dt = dt
        self.h = lib().orc_create(dt, seed)
        self.groups = []
        self.n_nodes = 0
        self._pending = []      # groups are added lazily so params can be edited

    def __del__(self):
        try:
            if self.h:
                lib().orc_free(self.h)
        except Exception:
            pass

    def create(self, model, n, n_port=0, params=None, vars=None, h_min_rel=1e-3,
               h0_rel=1e-2, eps=1e-6):
        """params / vars: dict name -> scalar, per-port list, or per-neuron array."""
        sv, svd, pv, pvd, sp, spd, pp, ppd = MODELS[model]
        if model in (AEIF_PSC_DELTA, IAF_PSC_EXP_G, IZHIKEVICH, IZH_PSC_EXP):
            n_port = 1
        nvar = len(sv) + len(pv) * n_port
        nparam = len(sp) + len(pp) * n_port
        V = np.zeros((n, max(nvar, 1)))
        P = np.zeros((n, max(nparam, 1)))
        for j, d in enumerate(svd):
            V[:, j] = d
        for q in range(n_port):
            for k, d in enumerate(pvd):
                V[:, len(sv) + q * len(pv) + k] = d
        for j, d in enumerate(spd):
            P[:, j] = d
        for q in range(n_port):
            for k, d in enumerate(ppd):
                P[:, len(sp) + q * len(pp) + k] = d
        if model == IZH_COND_BETA and "u" not in (vars or {}):
            b = (params or {}).get("b", 0.2)
            V[:, 1] = b * V[:, 0]

        def assign(M, names_s, names_p, d):
            for k, v in (d or {}).items():
                if k in names_s:
                    M[:, names_s.index(k)] = v
                elif k in names_p:
                    arr = np.asarray(v, dtype=float)
                    for q in range(n_port):
                        col = len(names_s) + q * len(names_p) + names_p.index(k)
                        M[:, col] = arr[..., q] if arr.ndim else arr
                else:
                    raise KeyError(k)
        assign(V, sv, pv, vars)
        assign(P, sp, pp, params)
        V = np.ascontiguousarray(V, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        i0 = lib().orc_add_group(self.h, model, n, n_port, nvar, nparam, _ptr(P, _dp),
                                 _ptr(V, _dp), h_min_rel, h0_rel, eps)
        g = Group(self, model, n, n_port, i0, len(self.groups))
        self.groups.append(g)
        self.n_nodes += n
        return g

    def set_spikes(self, group, times_per_node, heights_per_node=None):
        """Spike generator tables; times in ms (rounded to steps like the
        reference, src/spike_generator.cu:236)."""
        off = [0]
        steps, heights = [], []
        for i, tl in enumerate(times_per_node):
            for k, t in enumerate(tl):
                steps.append(int(round(np.float32(t) / np.float32(self.dt))))
                heights.append(1.0 if heights_per_node is None else heights_per_node[i][k])
            off.append(len(steps))
        off = np.asarray(off, dtype=np.int32)
        steps = np.asarray(steps + [0], dtype=np.int32)
        heights = np.asarray(heights + [0.0], dtype=np.float64)
        lib().orc_set_spikes(self.h, group.gid, _ptr(off, _ip), _ptr(steps, _ip),
                             _ptr(heights, _dp))

    def syn_group(self, model, params):
        if model == "stdp":
            names = ["tau_plus", "tau_minus", "lambda", "alpha", "mu_plus", "mu_minus", "Wmax"]
            d = dict(zip(names, [20.0, 20.0, 1e-4, 1.0, 1.0, 1.0, 100.0]))
            t = 2
        else:
            names = ["fact", "offset"]
            d = {"fact": 0.1, "offset": 0.0}
            t = 1
        d.update(params or {})
        p = np.asarray([np.float32(d[k]) for k in names], dtype=np.float64)
        return lib().orc_add_syn_group(self.h, t, _ptr(p, _dp), len(names))

    def connect(self, src, tgt, port, weight, delay, syn=None):
        src = np.ascontiguousarray(src, dtype=np.int32)
        n = len(src)
        tgt = np.ascontiguousarray(tgt, dtype=np.int32)
        port = np.ascontiguousarray(np.broadcast_to(port, (n,)), dtype=np.int32)
        syn = np.ascontiguousarray(np.broadcast_to(0 if syn is None else syn, (n,)), dtype=np.int32)
        w = np.ascontiguousarray(np.broadcast_to(weight, (n,)), dtype=np.float32)
        d = np.ascontiguousarray(np.broadcast_to(delay, (n,)), dtype=np.float32)
        lib().orc_connect(self.h, n, _ptr(src, _ip), _ptr(tgt, _ip), _ptr(port, _ip),
                          _ptr(syn, _ip), _ptr(w, _fp), _ptr(d, _fp))

    def set_step_search(self, group, on=True):
        """Exact step search for an RK5 group: every sub-step takes the
        largest step the error test accepts (a lower bound on the stage
        evaluations of any step proposer)."""
        lib().orc_set_step_search(self.h, group.gid, 1 if on else 0)

    def group_evals(self, group):
        return lib().orc_group_evals(self.h, group.gid)

    def set_direct_streams(self, streams):
        """Random streams of the Poisson direct connections in their (source,
        delay, insertion) order, e.g. those a sample of neurons has in a
        larger network (the GPU numbers them the same way)."""
        st = np.ascontiguousarray(streams, dtype=np.uint64)
        lib().orc_set_direct_streams(self.h, len(st), st.ctypes.data_as(ctypes.c_void_p))

    def simulate(self, n_steps, record=()):
        """record: list of (node, var_index). Returns array [n_steps, len(record)]."""
        nodes = np.asarray([r[0] for r in record] + [0], dtype=np.int32)
        cols = np.asarray([r[1] for r in record] + [0], dtype=np.int32)
        out = np.zeros((n_steps, max(len(record), 1)), dtype=np.float64)
        lib().orc_simulate(self.h, n_steps, len(record), _ptr(nodes, _ip), _ptr(cols, _ip),
                           _ptr(out, _dp))
        return out[:, :len(record)]

    def flush(self):
        lib().orc_flush(self.h)

    def spikes(self):
        n = lib().orc_n_spikes(self.h)
        steps = np.zeros(max(n, 1), dtype=np.int64)
        nodes = np.zeros(max(n, 1), dtype=np.int32)
        lib().orc_get_spikes(self.h, _ptr(steps, _llp), _ptr(nodes, _ip))
        return steps[:n], nodes[:n]

    def weights(self, n_edges):
        w = np.zeros(max(n_edges, 1), dtype=np.float32)
        lib().orc_get_weights(self.h, _ptr(w, _fp))
        return w[:n_edges]

    def state(self, node, nvar, nparam=0):
        v = np.zeros(max(nvar, 1))
        p = np.zeros(max(nparam, 1))
        lib().orc_get_state(self.h, node, _ptr(v, _dp), _ptr(p, _dp) if nparam else None)
        return v[:nvar], p[:nparam]

    def stage_evals(self):
        return lib().orc_stage_evals(self.h)
