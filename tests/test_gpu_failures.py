"""Failure handling on the device, without faulting the GPU.

Every device wait in the engine is bounded.  The self-test kernel waits at the
engine's grid barrier for a CTA that never arrives: the wait must give up on
its own, report the barrier status bit, and leave the context usable for the
next solve.
"""
import pytest

import mrcuda
from mrcuda import workloads as W

pytestmark = pytest.mark.gpu

STATUS_BARRIER = 1 << 4


def test_barrier_wait_times_out_and_the_context_survives():
    eng = mrcuda.Engine(0)
    for spins in (1, 1000, 20000):
        out = eng.selftest_wait_timeout(spins)
        assert out["status"] & STATUS_BARRIER, out
        assert out["ms"] < 2000.0
    wl = W.plain_board(n_nets=4)
    got = eng.route_isolated_batch(wl.request())
    assert all(p is not None for p in got.paths)
    eng.close()


def test_busy_engine_refuses_instead_of_waiting():
    """NO_WAIT on a context whose lock is taken fails at once with Busy (the
    reference's try_lock contract, cli/src/lib.rs:620-622)."""
    import threading

    eng = mrcuda.Engine(0)
    wl = W.congestion_board(seed=5, w=384, h=384, layers=4, n_nets=64)
    req = wl.request()
    started, busy_seen = threading.Event(), []

    def long_call():
        started.set()
        for _ in range(4):
            eng.route_isolated_batch(req)

    th = threading.Thread(target=long_call)
    th.start()
    started.wait()
    small = W.plain_board(n_nets=2).request()
    for _ in range(2000):
        try:
            eng.route_isolated_batch(small, no_wait=True)
        except mrcuda.Busy:
            busy_seen.append(True)
            break
        if not th.is_alive():
            break
    th.join()
    if not busy_seen:
        pytest.skip("the long call finished before a contended attempt")
    # after the contention the engine serves normally
    assert eng.route_isolated_batch(small).paths[0] is not None
    eng.close()
