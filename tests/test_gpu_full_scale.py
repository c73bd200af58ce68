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
