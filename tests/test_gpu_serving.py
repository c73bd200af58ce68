"""The continuous-batching request loop (mrc_server_*).

Each request's result must be the same bit for bit whether it is solved alone
(mrc_route_isolated_batch) or merged with others into shared launches, with
several launches in flight, under a tight memory budget, or one at a time, and
equal the CPU oracle's answer for the same request.
"""
import threading

import numpy as np
import pytest

import mrcuda
from mrcuda import workloads as W
from mrcuda.types import Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

from test_gpu_parity import _random_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = mrcuda.Engine(0)
    yield e
    e.close()


def _mixed_requests(n=24, seed=31):
    rng = np.random.default_rng(seed)
    reqs = []
    pool = [W.congestion_board(seed=100 + k, w=int(rng.integers(64, 200)), h=int(rng.integers(64, 200)),
                               layers=int(rng.integers(2, 7)), n_nets=0) for k in range(4)]
    tr = W.serving_trace(pool, 100.0, n // 2, seed=seed, min_nets=4, max_nets=40)
    reqs += [wl.request() for _, wl in tr]
    trial = 0
    while len(reqs) < n:
        r = _random_case(rng, trial, directed=trial % 2 == 0, max_side=60, max_layers=6)
        trial += 1
        if r is not None:
            reqs.append(r)
    order = rng.permutation(len(reqs))
    return [reqs[i] for i in order]


def _alone(engine, reqs, keep=False):
    return [engine.route_isolated_batch(r, retry_full=True, keep_fields=keep) for r in reqs]


def _same(a, b):
    assert a.paths == b.paths
    assert a.search_costs == b.search_costs
    assert a.retried == b.retried
    if a.fields is not None or b.fields is not None:
        assert len(a.fields) == len(b.fields)
        for x, y in zip(a.fields, b.fields):
            np.testing.assert_array_equal(x, y)


def _submit_all(srv, reqs, threads=4, keep=False):
    tickets = [None] * len(reqs)

    def worker(k):
        for i in range(k, len(reqs), threads):
            tickets[i] = srv.submit(reqs[i], retry_full=True, keep_fields=keep)

    ts = [threading.Thread(target=worker, args=(k,)) for k in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return [srv.wait(t) for t in tickets]


_ORACLE_CACHE = {}


def _oracle_results(oracle, reqs, key):
    """The oracle's (paths, costs) per request, with the full-board retry."""
    if key not in _ORACLE_CACHE:
        _ORACLE_CACHE[key] = [oracle.isolated_batch(r, retry_full=True, mode="field") for r in reqs]
    return _ORACLE_CACHE[key]


@pytest.mark.parametrize("slots,max_batch", [(2, 64), (3, 5), (1, 1)])
def test_same_result_alone_and_in_the_mix(engine, oracle, slots, max_batch):
    reqs = _mixed_requests()
    exp = _oracle_results(oracle, reqs, "mixed-24-31")
    alone = _alone(engine, reqs)
    srv = engine.server(slots=slots, max_batch_requests=max_batch)
    got = _submit_all(srv, reqs)
    for (res, info), ref, (ep, ec) in zip(got, alone, exp):
        _same(res, ref)
        assert res.paths == ep and res.search_costs == ec
        assert info["status"] == 0 and info["total_ms"] >= info["run_ms"] >= 0
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    if max_batch == 1:
        assert st["launches"] == len(reqs) and st["largest_launch"] == 1
    srv.close()


def test_fields_and_flags_groups(engine):
    """Requests asking for fields are batched apart from the others; both are exact."""
    reqs = _mixed_requests(12, seed=7)
    alone_f = _alone(engine, reqs, keep=True)
    srv = engine.server(slots=2)
    t1 = [srv.submit(r, keep_fields=True) for r in reqs]
    t2 = [srv.submit(r, retry_full=False) for r in reqs]
    for t, ref in zip(t1, alone_f):
        _same(srv.wait(t)[0], ref)
    for t, r in zip(t2, reqs):
        ref = engine.route_isolated_batch(r, retry_full=False)
        res = srv.wait(t)[0]
        assert res.paths == ref.paths and res.search_costs == ref.search_costs
    srv.close()


def test_memory_admission(engine):
    """A budget that holds only a few requests at a time still completes every
    request exactly; a request larger than the whole budget fails alone."""
    reqs = _mixed_requests(16, seed=9)
    alone = _alone(engine, reqs)
    srv = engine.server(slots=2, hbm_fraction=0.8)
    budget = srv.stats()["budget_bytes"]
    srv.close()
    # a fraction that leaves about 150 MB above what is already in use (the
    # budget counts the engine's own free pool blocks as available, so "in use"
    # is 0.8 * total - budget, not what the driver reports as taken)
    import torch

    _, t = torch.cuda.mem_get_info()
    frac = (0.8 * t - budget + 150e6) / t
    srv = engine.server(slots=2, hbm_fraction=frac)
    small = srv.stats()["budget_bytes"]
    assert 0 < small < budget
    got = _submit_all(srv, reqs, threads=2)
    for (res, _), ref in zip(got, alone):
        _same(res, ref)
    st = srv.stats()
    assert st["peak_bytes"] <= small
    big = W.congestion_board(seed=3, w=1024, h=1024, layers=4, n_nets=200).request()
    tk = srv.submit(big)
    with pytest.raises(mrcuda.LimitExceeded):
        srv.wait(tk)
    # the server keeps serving after the refusal
    res, _ = srv.wait(srv.submit(reqs[0]))
    _same(res, alone[0])
    srv.close()


def test_submit_validation_and_unknown_tickets(engine):
    srv = engine.server()
    dims = Dims(5, 3)
    bad = IsolatedRouteRequest(Grid.filled(dims, 1), [NetEndpoints("x", 0, 99)], [IsolatedRouteWindow.full(dims)],
                               [1] * 4, [1] * 2, [])
    with pytest.raises(mrcuda.InvalidEndpoint):
        srv.submit(bad)
    too_deep = IsolatedRouteRequest(Grid.filled(Dims(4, 4, 12), 1), [NetEndpoints("d", 0, 1)],
                                    [IsolatedRouteWindow(0, 0, 3, 3)], [1] * 3, [1] * 3, [1] * 11)
    with pytest.raises(mrcuda.LimitExceeded):
        srv.submit(too_deep)
    with pytest.raises(mrcuda.InvalidArgument):
        srv.wait(123456)
    empty = IsolatedRouteRequest(Grid.filled(dims, 1), [], [], [1] * 4, [1] * 2, [])
    res, info = srv.wait(srv.submit(empty))
    assert res.paths == [] and info["status"] == 0
    srv.close()


def test_resident_boards_mixed_with_uploaded_ones(engine, oracle):
    """Requests against boards kept in HBM and requests that bring their own
    board share launches; every result equals the request solved alone and the
    oracle's answer."""
    pool = [W.congestion_board(seed=200 + k, w=96 + 40 * k, h=80 + 30 * k, layers=2 + k, n_nets=0) for k in range(3)]
    boards = [engine.board(b.grid, b.x, b.y, b.vias, b.directed) for b in pool]
    trace = W.serving_trace(pool, 50.0, 30, seed=4, min_nets=4, max_nets=48)
    srv = engine.server(slots=3, max_batch_requests=16)
    tickets = []
    for i, (_, wl) in enumerate(trace):
        if i % 2:
            tickets.append(srv.submit_resident(boards[wl.meta["board_index"]], wl.nets, wl.windows))
        else:
            tickets.append(srv.submit(wl.request()))
    for t, (_, wl) in zip(tickets, trace):
        res, _ = srv.wait(t)
        _same(res, engine.route_isolated_batch(wl.request()))
        ep, ec = oracle.isolated_batch(wl.request(), retry_full=True, mode="field")
        assert res.paths == ep and res.search_costs == ec
    assert srv.stats()["largest_launch"] >= 1
    srv.close()
    for b in boards:
        b.close()
