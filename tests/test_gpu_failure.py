"""Bounded device waits: a wait that runs out ends the call with
MCE_ETIMEOUT; the kernel returns, so the handle and the device stay usable.
The wait is made to run out by giving it no work (no subtree is ever
shared) and a 1 ms limit - no fault, trap or endless loop is involved."""
import pytest

import mce_b200 as mce
import oracle

pytestmark = pytest.mark.gpu


def test_idle_wait_limit_times_out_and_handle_stays_usable():
    g = mce.gen_er(220, 0.5, 1)  # dense: the heaviest root walks ~4e4 tree nodes on one warp
    want = oracle.count(g)[0]
    with mce.Graph.from_host(g) as dg:
        # donation never starts: the warps without a root wait for subtrees
        # that never come while the heaviest trees run far longer than 1 ms
        with pytest.raises(mce.MceError) as e:
            dg.count(donate_after=1 << 30, wait_limit_ms=1)
        assert e.value.code == mce.ETIMEOUT
        r = dg.count()                      # the same handle, default limit
        r2 = dg.count(donate_after=1 << 30)  # and the starved schedule, default limit
    assert r.total == want and r2.total == want
