"""Device-side connection builder against the oracle's restatement of the
connection rules. Needs a B200.

Every rule call draws from the same counter-based streams on both sides, so
the graph must be identical edge for edge: the library's connections, in its
(source, delay, insertion) order, equal the oracle's insertion-order list
after a stable sort by (source, delay)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _expected(calls, dt=0.1):
    """calls: list of (rule, call index, sources, targets, param, weight,
    delay ms, port) -> arrays in delivery order."""
    from oracle import oracle as orc
    S, T, W, D, P = [], [], [], [], []
    for rule, call, src, tgt, param, w, d, port in calls:
        si, ti = orc.rule_edges(rule, 4242, call, len(src), len(tgt), param)
        S.append(np.asarray(src)[si])
        T.append(np.asarray(tgt)[ti])
        W.append(np.broadcast_to(np.asarray(w, dtype=np.float32), si.shape))
        D.append(np.full(len(si), int(round(np.float32(d) / np.float32(dt)))))
        P.append(np.full(len(si), port))
    S, T, W, D, P = (np.concatenate(x) for x in (S, T, W, D, P))
    order = np.lexsort((D, S))           # stable: insertion order inside
    return S[order], T[order], W[order], D[order], P[order]


def _check(ngpu, calls):
    s, t, w, d, p = _expected(calls)
    c = ngpu.GetAllConnections()
    assert len(c["source"]) == len(s)
    assert np.array_equal(c["source"], s)
    assert np.array_equal(c["target"], t)
    assert np.array_equal(c["port"], p)
    assert np.array_equal(np.rint(c["delay"] / 0.1).astype(int), d)
    assert np.array_equal(c["weight"], w)


def test_rules_match_oracle(ngpu):
    ngpu.SetRandomSeed(4242)
    a = ngpu.Create("aeif_cond_beta", 300, 2)
    b = ngpu.Create("aeif_cond_beta", 500, 2)
    pa, pb = list(range(a.i0, a.i0 + 300)), list(range(b.i0, b.i0 + 500))
    odd = pb[1::2]                                   # an explicit, non-contiguous list
    calls = []
    ngpu.Connect(a, b, {"rule": "fixed_indegree", "indegree": 40},
                 {"weight": 0.5, "delay": 2.0, "receptor": 0})          # rejection sampling
    calls.append(("fixed_indegree", 0, pa, pb, 40, 0.5, 2.0, 0))
    ngpu.Connect(a[0:50], odd, {"rule": "fixed_indegree", "indegree": 20},
                 {"weight": 0.25, "delay": 1.0, "receptor": 1})         # Fisher-Yates (pool < 5 K)
    calls.append(("fixed_indegree", 1, pa[0:50], odd, 20, 0.25, 1.0, 1))
    ngpu.Connect(b, a, {"rule": "fixed_outdegree", "outdegree": 7},
                 {"weight": 0.125, "delay": 3.0, "receptor": 0})
    calls.append(("fixed_outdegree", 2, pb, pa, 7, 0.125, 3.0, 0))
    ngpu.Connect(a, a, {"rule": "fixed_total_number", "total_num": 5000},
                 {"weight": 1.5, "delay": 1.0, "receptor": 1})
    calls.append(("fixed_total_number", 3, pa, pa, 5000, 1.5, 1.0, 1))
    ngpu.Connect(a[0:10], b[0:20], {"rule": "all_to_all"},
                 {"weight": 2.0, "delay": 0.5, "receptor": 0})
    calls.append(("all_to_all", 4, pa[0:10], pb[0:20], 0, 2.0, 0.5, 0))
    warr = (np.arange(100) * 0.01).astype(np.float32)
    ngpu.Connect(a[0:100], b[0:100], {"rule": "one_to_one"},
                 {"weight": {"array": warr.tolist()}, "delay": 1.0, "receptor": 0})
    calls.append(("one_to_one", 5, pa[0:100], pb[0:100], 0, warr, 1.0, 0))
    _check(ngpu, calls)
    # single connections keep their place in insertion order
    ngpu.SingleConnect(a[3], b[7], 0, 9.0, 1.0)
    s, t, w, d, p = _expected(calls)
    c = ngpu.GetAllConnections()
    assert len(c["source"]) == len(s) + 1
    k = np.nonzero((c["source"] == a[3]) & (c["target"] == b[7]) & (c["weight"] == 9.0))[0]
    assert len(k) == 1
    ngpu.Simulate(1.0)                                # calibration after the queries
    assert ngpu.NConnections() == len(s) + 1


def test_large_fixed_indegree_matches_oracle(ngpu):
    """1e7 synapses (50,000 targets x 200 sources each, two delays)."""
    ngpu.SetRandomSeed(4242)
    n = 50000
    pop = ngpu.Create("aeif_cond_beta", n, 2)
    ids = list(range(pop.i0, pop.i0 + n))
    ngpu.Connect(pop, pop, {"rule": "fixed_indegree", "indegree": 100},
                 {"weight": 0.1, "delay": 1.0, "receptor": 0})
    ngpu.Connect(pop, pop, {"rule": "fixed_indegree", "indegree": 100},
                 {"weight": 0.2, "delay": 2.0, "receptor": 1})
    _check(ngpu, [("fixed_indegree", 0, ids, ids, 100, 0.1, 1.0, 0),
                  ("fixed_indegree", 1, ids, ids, 100, 0.2, 2.0, 1)])


def test_rule_errors(ngpu):
    a = ngpu.Create("aeif_cond_beta", 10, 2)
    with pytest.raises(ValueError):
        ngpu.Connect(a, a, {"rule": "fixed_indegree", "indegree": 11}, {"weight": 1.0, "delay": 1.0})
    with pytest.raises(ValueError):
        ngpu.Connect(a, a, {"rule": "all_to_all"}, {"weight": 1.0, "delay": 0.01})
    assert ngpu.NConnections() == 0
    ngpu.Connect(a, a, {"rule": "one_to_one"}, {"weight": 1.0, "delay": 1.0, "receptor": 5})
    with pytest.raises(ValueError):
        ngpu.Simulate(1.0)                            # port 5 does not exist
