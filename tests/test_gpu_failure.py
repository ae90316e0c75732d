"""Failure detection on the GPU without a GPU fault.

Every device-side wait of the library (the decoupled look-backs of the scans)
polls a bounded number of times; when it gives up it records FMCS_E_TIMEOUT in
the context's status word and lets its kernel finish, so the host reads an
error code and the context keeps working.  fmcs_selftest_wait runs that same
wait on a word that nothing writes: the wait must run out after the given
number of polls.  Nothing here traps, asserts or waits without a bound."""
import numpy as np
import pytest

from fastmulticolsort_b200 import capi
from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("polls", [1, 64, 4096])
def test_bounded_wait_times_out_and_context_recovers(polls):
    with capi.Context(0) as ctx:
        assert ctx.selftest_wait(polls) == capi.FMCS_E_TIMEOUT
        assert "timed out" in ctx._L.fmcs_last_error(ctx.handle).decode()
        # the status word was cleared: the same context sorts correctly next
        cols, bw = W.cols_17b33(1 << 18, seed_index=21)
        n = cols[0].shape[0]
        order = np.zeros(n, np.uint32)
        group = np.zeros(n, np.uint32)
        ng = ctx.run_plan(cols, bw, [50], order, group)
        o, g, ng_ref = O.run_plan_sort(cols, bw, [50])
        assert ng == ng_ref and np.array_equal(order, o) and np.array_equal(group, g)
        # and a second timeout is reported again
        assert ctx.selftest_wait(polls) == capi.FMCS_E_TIMEOUT


def test_selftest_rejects_bad_limits():
    with capi.Context(0) as ctx:
        assert ctx.selftest_wait(0) == capi.FMCS_E_INVAL
        assert ctx.selftest_wait((1 << 20) + 1) == capi.FMCS_E_INVAL
