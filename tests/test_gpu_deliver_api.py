"""NGB200_DeliverSpikes through the C ABI: one batch of spikes through a
random CSR graph, checked bit-exactly against the integer sum computed on
the host (fixed point with 32 fractional bits, the delivery's contract)."""
import ctypes

import numpy as np
import pytest

from neurongpu_b200 import LIB_PATH

pytestmark = pytest.mark.gpu


def make_case(rng, n_src=3000, nd=7, n_slots=5000, mean_deg=40, n_spikes=4000):
    deg = rng.poisson(mean_deg, size=n_src * nd).astype(np.uint64)
    deg[rng.random(n_src * nd) < 0.3] = 0            # empty groups
    grp_off = np.zeros(n_src * nd + 1, dtype=np.uint64)
    grp_off[1:] = np.cumsum(deg)
    E = int(grp_off[-1])
    e_slot = rng.integers(0, n_slots, size=E).astype(np.uint32)
    e_w = rng.choice(np.float32([0.05, 0.35, -0.125, 1.5, 87.8]), size=E).astype(np.float32)
    src = rng.integers(0, n_src, size=n_spikes).astype(np.uint32)
    h = rng.choice(np.float32([1.0, 2.0, 0.5]), size=n_spikes).astype(np.float32)
    di = rng.integers(0, nd, size=n_spikes).astype(np.int32)
    return grp_off, e_slot, e_w, nd, src, h, di, n_slots


def host_reference(grp_off, e_slot, e_w, nd, src, h, di, n_slots):
    acc = np.zeros(n_slots, dtype=np.int64)
    for s, hh, d in zip(src, h, di):
        g = int(s) * nd + int(d)
        b, e = int(grp_off[g]), int(grp_off[g + 1])
        if b == e:
            continue
        v = (np.float32(hh) * e_w[b:e]).astype(np.float64)
        np.add.at(acc, e_slot[b:e], np.rint(v * 2.0 ** 32).astype(np.int64))
    return acc


def device_call(fn_name, case):
    import torch
    grp_off, e_slot, e_w, nd, src, h, di, n_slots = case
    lib = ctypes.CDLL(LIB_PATH)
    fn = getattr(lib, fn_name)
    fn.restype = ctypes.c_int
    t = {k: torch.from_numpy(v.astype(v.dtype)).cuda() for k, v in
         dict(grp_off=grp_off.view(np.int64), e_slot=e_slot.view(np.int32), e_w=e_w,
              src=src.view(np.int32), h=h, di=di).items()}
    acc = torch.zeros(n_slots, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    rc = fn(p(t["grp_off"]), p(t["e_slot"]), p(t["e_w"]), ctypes.c_int(nd), p(t["src"]),
            p(t["h"]), p(t["di"]), ctypes.c_int(len(src)), p(acc), ctypes.c_void_p(0))
    torch.cuda.synchronize()
    return rc, acc.cpu().numpy()


def test_deliver_spikes_matches_host_integer_sum():
    rng = np.random.default_rng(3)
    case = make_case(rng)
    rc, acc = device_call("NGB200_DeliverSpikes", case)
    assert rc == 0
    ref = host_reference(*case)
    assert np.count_nonzero(ref) > 1000
    np.testing.assert_array_equal(acc, ref)


def test_deliver_spikes_rejects_bad_delay_index():
    rng = np.random.default_rng(4)
    case = list(make_case(rng, n_spikes=10))
    case[6] = case[6].copy()
    case[6][3] = case[3]            # di == nd is out of range
    rc, _ = device_call("NGB200_DeliverSpikes", tuple(case))
    assert rc == 4
