"""Host-side checks of the device error paths that a GPU test cannot force
safely: the parity bookkeeping that the step proposer's tensor-core rounds
use to find the completion still pending after a timed-out wait. No compute
call is made.

An mbarrier completes phases 0, 1, 2, ... in order; a wait on parity P
succeeds once the most recent phase with parity P has completed. The model
below tracks the number of completed phases and checks, for every outcome
of a round, that the parity the round keeps names the right completion:
the pending one after a failed wait (the teardown must block until it
lands, then see it), the next round's first one after a complete round.
"""
import itertools

import pytest


class Barrier(object):
    def __init__(self, completed):
        self.completed = completed     # phases completed so far

    def wait_ok(self, parity):
        # the phase being waited for is the first incomplete phase with this
        # parity or the last completed one; it has completed iff the current
        # (incomplete) phase has the other parity
        return (self.completed & 1) != parity

    def complete(self):
        self.completed += 1


@pytest.mark.parametrize("start,ok1,ok2", list(itertools.product((0, 1, 2, 7), (True, False),
                                                                 (True, False))))
def test_proposer_phase_bookkeeping(start, ok1, ok2):
    from neurongpu_b200 import neurongpu as api
    b = api.default_binding()
    bar = Barrier(start)
    ph0 = start & 1                    # parity of the round's first completion
    # layer 1 committed; its wait succeeds iff it completed in time
    if ok1:
        bar.complete()
        assert bar.wait_ok(ph0)
        # layer 2 committed
        if ok2:
            bar.complete()
            assert bar.wait_ok(ph0 ^ 1)
    else:
        assert not bar.wait_ok(ph0)
    kept = b.ProposerPhaseAfter(ph0, ok1, ok2)
    if ok1 and ok2:
        # the next round's first completion: not complete yet, and it is
        # the one that the next commit completes
        assert not bar.wait_ok(kept)
        bar.complete()
        assert bar.wait_ok(kept)
    else:
        # teardown after a failure: the kept parity must still be pending
        # (an immediate success would release the tensor memory under a
        # running MMA) and must succeed once the pending completion lands
        assert not bar.wait_ok(kept)
        bar.complete()
        assert bar.wait_ok(kept)
