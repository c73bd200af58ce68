"""Snapshot negotiation rounds on the device vs the CPU snapshot oracle.

Every round must agree exactly: the dirty set, every net's path, the price
snapshot, the per-edge occupancy and history, and the round statistics.
"""
import numpy as np
import pytest

import mrcuda
from mrcuda import workloads as W
from mrcuda.types import Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

from snapshot_oracle import SnapshotNegotiation

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[1, 2], ids=["cta-tiles", "warp-tiles"])
def engine(request):
    """Every test runs on both default schedules: a CTA per tile and a warp per tile."""
    e = mrcuda.Engine(0)
    e.set_schedule(request.param)
    yield e
    e.close()


def _run_both(engine, oracle, req, rounds, weight=16, step=1, check_arrays=True, groups=None, clearance=0,
              via_keepout=0):
    dev = engine.negotiation(req, present_weight=weight, history_step=step, groups=groups, clearance=clearance,
                             via_keepout=via_keepout)
    cpu_groups = mrcuda.connection_group_ids(req.nets) if groups == "connections" else groups
    cpu = SnapshotNegotiation(oracle, req, present_weight=weight, history_step=step, groups=cpu_groups,
                              clearance=clearance, via_keepout=via_keepout)
    history = []
    for r in range(rounds):
        a = dev.round()
        b = cpu.round()
        assert a["dirty"] == b["dirty"], (r, a, b)
        if not b["dirty"]:
            break
        for k in ("pfac", "routed", "overused_edges", "next_dirty"):
            assert a[k] == b[k], (r, k, a, b)
        assert dev.paths() == cpu.paths, r
        assert dev.dirty() == cpu.dirty, r
        if check_arrays:
            present, hist, snap = dev.read()
            np.testing.assert_array_equal(present, cpu.present, err_msg=f"present, round {r}")
            np.testing.assert_array_equal(hist, cpu.history, err_msg=f"history, round {r}")
            np.testing.assert_array_equal(snap, cpu.snapshot, err_msg=f"snapshot, round {r}")
            if clearance or via_keepout:
                np.testing.assert_array_equal(dev.read_halo(), cpu.halo, err_msg=f"halo, round {r}")
        history.append(a)
    dev.close()
    return history


def test_rounds_match_the_oracle_on_a_congested_board(engine, oracle):
    wl = W.snapshot_board(w=160, h=128, layers=3, n_nets=80, median=60)
    hist = _run_both(engine, oracle, wl.request(), rounds=8)
    assert hist[0]["overused_edges"] > 0 and hist[-1]["dirty"] < hist[0]["dirty"]
    assert all(h["round_ms"] > 0 for h in hist)


def test_axis_prices_own_pads_and_other_weights(engine, oracle):
    """Base prices from the per-axis vectors, obstacles, own pads, a zero
    history step and a large congestion weight."""
    wl = W.plain_board(seed=21, w=96, h=80, layers=2, n_nets=40)
    req = wl.request()
    rng = np.random.default_rng(5)
    nets = []
    for nt in req.nets:
        pads = sorted({int(c) for c in rng.integers(0, len(req.grid.dims), 2)})
        nets.append(NetEndpoints(nt.net, nt.src, nt.dst, pads))
    req = IsolatedRouteRequest(req.grid, nets, [mrcuda.net_windows(req.grid.dims, [n])[0] for n in nets],
                               rng.integers(1, 20, 95).astype(np.uint32), rng.integers(1, 20, 79).astype(np.uint32),
                               [7])
    _run_both(engine, oracle, req, rounds=5, weight=200, step=0)
    _run_both(engine, oracle, req, rounds=5, weight=1, step=5)


def test_windows_that_need_the_retry(engine, oracle):
    """Tight windows around a wall: the retry runs on the snapshot board."""
    dims = Dims(40, 20, 2)
    cost = np.ones((2, 20, 40), np.uint32)
    cost[:, 0:18, 20] = 0xFFFFFFFF
    grid = Grid(dims, cost.reshape(-1))
    nets = [NetEndpoints(f"w{i}", dims.idx3(2 + i, 2 + i, 0), dims.idx3(37 - i, 3 + i, i % 2)) for i in range(8)]
    wins = [IsolatedRouteWindow(0, 0, 39, 12)] * len(nets)
    req = IsolatedRouteRequest(grid, nets, wins, [10] * 39, [10] * 19, [30])
    hist = _run_both(engine, oracle, req, rounds=6)
    assert hist[0]["retried"] == len(nets)


def test_converged_rounds_do_nothing(engine, oracle):
    dims = Dims(30, 30, 1)
    grid = Grid.filled(dims, 1)
    nets = [NetEndpoints("a", dims.idx(1, 1), dims.idx(10, 1)), NetEndpoints("b", dims.idx(1, 20), dims.idx(10, 20))]
    req = IsolatedRouteRequest(grid, nets, [IsolatedRouteWindow.full(dims)] * 2, [10] * 29, [10] * 29, [])
    neg = engine.negotiation(req)
    first = neg.round()
    assert first["dirty"] == 2 and first["overused_edges"] == 0 and first["next_dirty"] == 0
    paths = neg.paths()
    again = neg.round()
    assert again["dirty"] == 0 and neg.paths() == paths
    neg.close()


def test_medium_board_rounds(engine, oracle):
    """512x512x4, 300 nets, 4 rounds: paths, statistics and arrays."""
    wl = W.snapshot_board(seed=8, w=512, h=512, layers=4, n_nets=300, median=120)
    _run_both(engine, oracle, wl.request(), rounds=4)


def test_connection_groups_on_a_congested_board(engine, oracle):
    """Group-aware overuse: nets renamed into "#"-sibling groups of eight (and
    groups by shared endpoints), every round against the oracle; then explicit
    ids.  Same-group sharing adds no history, so the rounds differ from the
    ungrouped ones."""
    wl = W.snapshot_board(w=160, h=128, layers=3, n_nets=80, median=60)
    req = wl.request()
    nets = [NetEndpoints(f"g{i // 8}#{i % 8}", nt.src, nt.dst, nt.passable_pads, nt.via_passable_pads)
            for i, nt in enumerate(req.nets)]
    req = IsolatedRouteRequest(req.grid, nets, req.windows, req.x_edge_costs, req.y_edge_costs, req.via_edge_costs,
                               req.directed_in_costs)
    grouped = _run_both(engine, oracle, req, rounds=6, groups="connections")
    plain = _run_both(engine, oracle, req, rounds=6)
    assert grouped[0]["overused_edges"] < plain[0]["overused_edges"]  # same-group sharing is free
    _run_both(engine, oracle, req, rounds=4, groups=[i % 5 for i in range(len(nets))])


def test_connection_groups_are_checked(engine):
    wl = W.snapshot_board(w=64, h=48, layers=2, n_nets=6, median=20)
    req = wl.request()
    with pytest.raises(mrcuda.InvalidArgument):
        engine.negotiation(req, groups=[0] * 5)
    with pytest.raises(mrcuda.InvalidArgument):
        engine.negotiation(req, groups=[0xFFFFFFFF] * 6)
    neg = engine.negotiation(req)
    neg.round()
    g = np.zeros(6, np.uint32)
    with pytest.raises(mrcuda.InvalidArgument):  # only before the first round
        neg.engine._check(neg.engine.lib.mrc_negotiation_set_groups(neg.engine.ctx, neg.handle, g.ctypes.data))
    neg.close()
    shard = engine.negotiation(req, owned=[True] * 6)
    with pytest.raises(mrcuda.InvalidArgument):  # a shard sees only part of the paths
        shard.engine._check(shard.engine.lib.mrc_negotiation_set_groups(shard.engine.ctx, shard.handle,
                                                                        g.ctypes.data))
    shard.close()


# ---- clearance-halo pricing ------------------------------------------------------


def test_clearance_rounds_match_the_oracle(engine, oracle):
    """The reference's clearance-active iteration: every net routed every
    round against the snapshot of all current paths plus their footprints,
    each net priced with its own copper and footprint subtracted (per-net
    overrides on the device).  Paths, dirty sets, occupancy, history, the
    shared snapshot and the footprint counts match the oracle every round."""
    wl = W.snapshot_board(seed=4, w=96, h=80, layers=2, n_nets=24, median=30)
    hist = _run_both(engine, oracle, wl.request(), rounds=5, clearance=1, via_keepout=2)
    assert hist[0]["dirty"] == 24 and hist[1]["dirty"] == 24
    _run_both(engine, oracle, wl.request(), rounds=3, clearance=2, via_keepout=0)
    _run_both(engine, oracle, wl.request(), rounds=3, clearance=0, via_keepout=1)


def test_clearance_corridor_and_retry(engine, oracle):
    """A corridor both nets must share (overuse never clears: both stay
    dirty), and tight windows whose nets need the full-board retry, which then
    runs with the same per-net overrides."""
    dims = Dims(9, 5, 1)
    cost = np.full((5, 9), 0xFFFFFFFF, np.uint32)
    cost[:, 0] = 1
    cost[:, 8] = 1
    cost[2, :] = 1
    nets = [NetEndpoints("a", dims.idx(0, 0), dims.idx(8, 0)), NetEndpoints("b", dims.idx(0, 4), dims.idx(8, 4))]
    req = IsolatedRouteRequest(Grid(dims, cost.reshape(-1)), nets, [IsolatedRouteWindow.full(dims)] * 2, [10] * 8,
                               [10] * 4, [])
    hist = _run_both(engine, oracle, req, rounds=4, clearance=1)
    assert all(h["dirty"] == 2 for h in hist)
    dims = Dims(40, 20, 2)
    cost = np.ones((2, 20, 40), np.uint32)
    cost[:, 0:18, 20] = 0xFFFFFFFF
    nets = [NetEndpoints(f"w{i}", dims.idx3(2 + i, 2 + i, 0), dims.idx3(37 - i, 3 + i, i % 2)) for i in range(8)]
    wins = [IsolatedRouteWindow(0, 0, 39, 12)] * len(nets)
    req = IsolatedRouteRequest(Grid(dims, cost.reshape(-1)), nets, wins, [10] * 39, [10] * 19, [30])
    hist = _run_both(engine, oracle, req, rounds=4, clearance=1, via_keepout=1)
    assert hist[1]["retried"] == len(nets)


@pytest.mark.parametrize("schedule", [0, 3])
def test_clearance_on_the_staged_word_schedules(oracle, schedule):
    """The rounds form and the queue form without price planes patch the
    staged directed words with the per-net overrides."""
    e = mrcuda.Engine(0)
    try:
        e.set_schedule(schedule)
        wl = W.snapshot_board(seed=6, w=80, h=64, layers=3, n_nets=20, median=24)
        _run_both(e, oracle, wl.request(), rounds=4, clearance=1, via_keepout=1)
    finally:
        e.close()


def test_clearance_is_checked(engine):
    wl = W.snapshot_board(w=64, h=48, layers=2, n_nets=6, median=20)
    req = wl.request()
    with pytest.raises(mrcuda.InvalidArgument):
        engine.negotiation(req, clearance=256)
    neg = engine.negotiation(req)
    with pytest.raises(mrcuda.InvalidArgument):  # no clearance set
        neg.read_halo()
    neg.round()
    with pytest.raises(mrcuda.InvalidArgument):  # only before the first round
        neg.engine._check(neg.engine.lib.mrc_negotiation_set_clearance(neg.engine.ctx, neg.handle, 1, 0, 16))
    neg.close()
    with pytest.raises(mrcuda.InvalidArgument):  # a shard sees only part of the paths
        engine.negotiation(req, owned=[True] * 6, clearance=1)


def test_clearance_with_connection_groups(engine, oracle):
    """Clearance rounds with group-aware overuse: prices count every other
    net's copper and footprint, overuse counts groups (copper only)."""
    wl = W.snapshot_board(seed=11, w=96, h=72, layers=2, n_nets=24, median=28)
    req = wl.request()
    nets = [NetEndpoints(f"c{i // 4}#{i % 4}", nt.src, nt.dst, nt.passable_pads, nt.via_passable_pads)
            for i, nt in enumerate(req.nets)]
    req = IsolatedRouteRequest(req.grid, nets, req.windows, req.x_edge_costs, req.y_edge_costs, req.via_edge_costs,
                               req.directed_in_costs)
    _run_both(engine, oracle, req, rounds=4, groups="connections", clearance=1, via_keepout=1)
