"""NGB200_DeliverSpikesNoAlloc, the allocation-free delivery entry point.

It serves callers that cannot allocate device memory while they run (a host
whose allocator owns the device memory, or a loop that must not stall on the
synchronisation a cudaMalloc / cudaFree brings). It must give exactly the
accumulators of NGB200_DeliverSpikes, call after call, although every call
reuses the same static scratch. This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from neurongpu_b200 import LIB_PATH
from tests.test_gpu_deliver_api import device_call, make_case

pytestmark = pytest.mark.gpu


def test_no_alloc_matches_allocating_entry_point_twice():
    rng = np.random.default_rng(21)
    # two calls in a row with different batches: the second call must not
    # see anything left in the shared scratch by the first
    for case in (make_case(rng, nd=7, n_spikes=4000), make_case(rng, nd=3, n_spikes=2500)):
        rc_a, acc_a = device_call("NGB200_DeliverSpikes", case)
        rc_b, acc_b = device_call("NGB200_DeliverSpikesNoAlloc", case)
        assert rc_a == 0 and rc_b == 0
        assert np.count_nonzero(acc_a) > 500
        # integer fixed-point sums: the tolerance is exact equality
        np.testing.assert_array_equal(acc_b, acc_a)


def test_no_alloc_rejects_batches_beyond_its_scratch():
    rng = np.random.default_rng(22)
    case = make_case(rng, nd=15, n_spikes=70000)     # 16 * 70000 > 2**20 entries
    rc, acc = device_call("NGB200_DeliverSpikesNoAlloc", case)
    assert rc == 5
    assert not np.any(acc)
