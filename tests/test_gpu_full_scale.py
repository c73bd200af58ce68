"""Full benchmark sizes, checked against the oracle or through properties that
do not depend on size.

* all 4096 uneven instances, every path and cost against the oracle's search
  of that instance alone;
* the 2048x2048x6 negotiation board with 3000 nets: after each round the
  occupancy equals a recount of the current paths, history moved by exactly one
  step on the slots that were overused, every path is a legal walk between its
  endpoints, and a sample of the rerouted nets equals the oracle's search on the
  round's own price snapshot.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import mrcuda
from mrcuda import workloads as W
from mrcuda.types import IsolatedRouteRequest

from snapshot_oracle import edge_slots

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = mrcuda.Engine(0)
    yield e
    e.close()


def test_all_4096_uneven_instances_match_the_oracle(engine, oracle):
    s = W.uneven_instances()
    reqs = s.requests()
    got = engine.route_instances(reqs)
    with ThreadPoolExecutor(max_workers=16) as ex:
        exp = list(ex.map(lambda r: oracle.isolated_batch(r, retry_full=True, mode="astar", threads=1), reqs))
    bad = [k for k, (g, e) in enumerate(zip(got, exp)) if (g.paths, g.search_costs) != e]
    assert not bad, bad[:10]
    assert sum(p is not None for g in got for p in g.paths) >= 4090


def _legal_walk(path, dims):
    p = np.asarray(path, dtype=np.int64)
    a, b = p[:-1], p[1:]
    plane = dims.plane
    same = (a // plane) == (b // plane)
    d = np.abs(b - a)
    planar = same & ((d == 1) & ((np.minimum(a, b) % plane) % dims.w + 1 < dims.w) | (d == dims.w))
    via = (~same) & (d == plane)
    return bool((planar | via).all()) and len(set(path)) == len(path)


def test_full_size_negotiation_round_properties(engine, oracle):
    wl = W.snapshot_board()
    req = wl.request()
    dims = wl.grid.dims
    neg = engine.negotiation(req)
    prev_hist = np.zeros((len(dims), 4), np.uint32)
    for r in range(2):
        dirty = neg.dirty()
        st = neg.round()
        present, hist, snap = neg.read()
        paths = neg.paths()
        recount = np.zeros_like(present)
        for p in paths:
            if p:
                c, sl = edge_slots(p, dims.w, dims.plane)
                np.add.at(recount, (c, sl), 1)
        np.testing.assert_array_equal(present, recount, err_msg=f"round {r}")
        over = present >= 2
        np.testing.assert_array_equal(hist, prev_hist + over.astype(np.uint32), err_msg=f"round {r}")
        assert st["overused_edges"] == int(over.sum()) // 2
        for i, p in enumerate(paths):
            if p:
                assert p[0] == req.nets[i].src and p[-1] == req.nets[i].dst and _legal_walk(p, dims), i
        # a sample of this round's nets, searched alone on this round's snapshot
        for i in dirty[:: max(1, len(dirty) // 6)][:6]:
            one = IsolatedRouteRequest(req.grid, [req.nets[i]], [req.windows[i]], req.x_edge_costs, req.y_edge_costs,
                                       req.via_edge_costs, snap.reshape(-1))
            e_paths, _ = oracle.isolated_batch(one, retry_full=True, mode="astar")
            assert paths[i] == e_paths[0], (r, i)
        prev_hist = hist
    neg.close()


def test_full_board_retry_at_full_size(engine, oracle):
    """A window that cannot hold the path on the 2048x2048x6 board: the retry
    solves the whole 25.2 M-cell board, and its path equals the oracle's."""
    from mrcuda.types import COST_MAX, IsolatedRouteWindow, NetEndpoints

    wl = W.snapshot_board(n_nets=1)
    dims = wl.grid.dims
    cost = wl.grid.cost.reshape(dims.layers, dims.h, dims.w).copy()
    cost[:, 100:2048, 1024] = COST_MAX  # a wall on every layer with its gap at y < 100
    src, dst = dims.idx3(1000, 1500, 0), dims.idx3(1050, 1500, 0)
    cost.reshape(-1)[[src, dst]] = 1
    grid = type(wl.grid)(dims, cost.reshape(-1))
    net = NetEndpoints("r", src, dst)
    req = IsolatedRouteRequest(grid, [net], [IsolatedRouteWindow(900, 1400, 1150, 1600)], wl.x, wl.y, wl.vias,
                               wl.directed)
    got = engine.route_isolated_batch(req, retry_full=True)
    assert got.retried == 1 and got.paths[0] is not None
    exp_paths, exp_costs = oracle.isolated_batch(req, retry_full=True, mode="field")
    assert got.paths == exp_paths and got.search_costs == exp_costs
    assert min(dims.xy(c)[1] for c in got.paths[0]) < 100  # it went around through the gap
