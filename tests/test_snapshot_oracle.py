"""CPU checks of the snapshot negotiation oracle (no GPU).

The oracle's round is pinned here by hand-checkable boards: slot bookkeeping,
a corridor two nets must share (overuse can never clear, so history grows by
one step per round on exactly the corridor edges), a detour that negotiation
finds, and the occupancy invariant (present == recount of the current paths).
"""
import numpy as np

from mrcuda import workloads as W
from mrcuda.types import COST_MAX, Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

from snapshot_oracle import SnapshotNegotiation, base_prices, edge_slots


def _recount(neg):
    cnt = np.zeros_like(neg.present)
    for p in neg.paths:
        c, s = edge_slots(p or [], neg.dims.w, neg.dims.plane)
        np.add.at(cnt, (c, s), 1)
    return cnt


def test_edge_slots_of_a_path():
    dims = Dims(4, 3, 2)
    # (0,0,0) -> (1,0,0) -> (1,1,0) -> via -> (1,1,1) -> (0,1,1)
    p = [dims.idx3(0, 0, 0), dims.idx3(1, 0, 0), dims.idx3(1, 1, 0), dims.idx3(1, 1, 1), dims.idx3(0, 1, 1)]
    c, s = edge_slots(p, dims.w, dims.plane)
    got = sorted(zip(c.tolist(), s.tolist()))
    exp = sorted([(p[1], 1), (p[0], 2),      # +x step: b from -x, a from +x
                  (p[2], 0), (p[1], 3),      # +y step: b from -y, a from +y
                  (p[4], 2), (p[3], 1)])     # -x step: b from +x, a from -x
    assert got == exp


def test_base_prices_from_axis_vectors():
    dims = Dims(3, 2, 1)
    req = IsolatedRouteRequest(Grid.filled(dims, 1), [], [], [5, 6], [7], [])
    b = base_prices(req).reshape(2, 3, 4)
    assert b[0, 1].tolist() == [COST_MAX, 5, 6, 7]
    assert b[1, 2].tolist() == [7, 6, COST_MAX, COST_MAX]


def test_shared_corridor_accumulates_history(oracle):
    """A one-cell-wide corridor both nets must use: every round both nets are
    dirty again and each corridor edge gains exactly one history step."""
    dims = Dims(9, 5, 1)
    cost = np.full((5, 9), COST_MAX, np.uint32)
    cost[:, 0] = 1
    cost[:, 8] = 1
    cost[2, :] = 1  # corridor along y = 2
    grid = Grid(dims, cost.reshape(-1))
    nets = [NetEndpoints("a", dims.idx(0, 0), dims.idx(8, 0)), NetEndpoints("b", dims.idx(0, 4), dims.idx(8, 4))]
    req = IsolatedRouteRequest(grid, nets, [IsolatedRouteWindow.full(dims)] * 2, [10] * 8, [10] * 4, [])
    neg = SnapshotNegotiation(oracle, req, history_step=3)
    for r in range(4):
        st = neg.round()
        assert st["dirty"] == 2 and st["routed"] == 2 and st["next_dirty"] == 2
        assert st["overused_edges"] == 8  # the 8 corridor edges
        np.testing.assert_array_equal(neg.present, _recount(neg))
        corridor = [dims.idx(x, 2) for x in range(1, 9)]
        assert (neg.history[corridor, 1] == 3 * (r + 1)).all()


def test_negotiation_spreads_nets_and_keeps_the_invariant(oracle):
    wl = W.snapshot_board(w=120, h=96, layers=2, n_nets=50, median=50)
    neg = SnapshotNegotiation(oracle, wl.request())
    first = neg.round()
    assert first["overused_edges"] > 0
    np.testing.assert_array_equal(neg.present, _recount(neg))
    for _ in range(6):
        st = neg.round()
        np.testing.assert_array_equal(neg.present, _recount(neg))
        if not st["dirty"]:
            break
    assert st.get("overused_edges", 0) < first["overused_edges"]
    # the snapshot never prices a blocked base edge
    assert (neg.snapshot[neg.base == COST_MAX] == COST_MAX).all()


def _corridor_request(names):
    dims = Dims(9, 5, 1)
    cost = np.full((5, 9), COST_MAX, np.uint32)
    cost[:, 0] = 1
    cost[:, 8] = 1
    cost[2, :] = 1  # corridor along y = 2
    grid = Grid(dims, cost.reshape(-1))
    nets = [NetEndpoints(names[0], dims.idx(0, 0), dims.idx(8, 0)),
            NetEndpoints(names[1], dims.idx(0, 4), dims.idx(8, 4))]
    return dims, IsolatedRouteRequest(grid, nets, [IsolatedRouteWindow.full(dims)] * 2, [10] * 8, [10] * 4, [])


def test_connection_groups_follow_the_reference_rule():
    """The reference's grouping (negotiated.rs:929-989, pinned by its test
    route_exports_aligned_group_ids): '#'-siblings share a group, a foreign
    net is its own; nets that share an endpoint cell are one group too; ids are
    dense in order of first appearance."""
    from mrcuda import connection_group_ids, group_of

    assert group_of("g#0") == "g" and group_of("plain") == "plain" and group_of("a#b#c") == "a"
    nets = [NetEndpoints("g#0", 0, 7), NetEndpoints("g#1", 16, 23), NetEndpoints("foreign", 40, 47)]
    assert connection_group_ids(nets) == [0, 0, 1]
    nets = [NetEndpoints("a", 0, 5), NetEndpoints("b", 5, 9), NetEndpoints("c", 10, 11), NetEndpoints("d#x", 12, 13),
            NetEndpoints("d#y", 14, 15), NetEndpoints("e", 11, 20), NetEndpoints("f", 30, 30)]
    assert connection_group_ids(nets) == [0, 0, 1, 2, 2, 1, 3]
    assert connection_group_ids([]) == []


def test_same_group_nets_share_a_corridor_without_overuse(oracle):
    """Two nets of one connection group through a one-cell corridor: the edges
    are not overused, so no history accrues and no net is dirty after round 0
    (prices still count both nets, as in route_negotiated).  Nets of two groups
    on the same board overuse all 8 corridor edges every round."""
    dims, req = _corridor_request(["n#0", "n#1"])
    neg = SnapshotNegotiation(oracle, req, history_step=3, groups=[0, 0])
    st = neg.round()
    assert st["routed"] == 2 and st["overused_edges"] == 0 and st["next_dirty"] == 0
    assert (neg.history == 0).all()
    assert (neg.present[[dims.idx(x, 2) for x in range(1, 9)], 1] == 2).all()
    _, req2 = _corridor_request(["a", "b"])
    neg2 = SnapshotNegotiation(oracle, req2, history_step=3, groups=[0, 1])
    for r in range(3):
        st = neg2.round()
        assert st["overused_edges"] == 8 and st["next_dirty"] == 2
    # every net its own group is the default test (count >= 2)
    neg3 = SnapshotNegotiation(oracle, req2, history_step=3)
    for r in range(3):
        neg3.round()
    np.testing.assert_array_equal(neg3.history, neg2.history)


# ---- clearance-halo pricing (the reference's clearance-active iteration) ----

from snapshot_oracle import halo_footprint  # noqa: E402


def test_halo_footprint_boxes_vias_and_obstacles():
    """for_each_halo_cell on a uniform grid (negotiated.rs:3184-3271): a
    (2r+1)^2 box per path cell on its own layer, clipped to the board, base
    obstacles skipped, repeats kept; a via adds the keepout box on both layers."""
    dims = Dims(6, 5, 2)
    cost = np.ones(len(dims), np.uint32)
    cost[dims.idx3(3, 1, 0)] = COST_MAX
    path = [dims.idx3(0, 0, 0), dims.idx3(1, 0, 0)]
    h = halo_footprint(path, dims, cost, 1, 0)
    # (0,0): box x 0..1, y 0..1 = 4 cells; (1,0): x 0..2, y 0..1 = 6 cells
    assert h.size == 10
    cnt = np.bincount(h, minlength=len(dims))
    assert cnt[dims.idx3(0, 0, 0)] == 2 and cnt[dims.idx3(2, 1, 0)] == 1 and cnt[dims.idx3(2, 2, 0)] == 0
    path = [dims.idx3(2, 1, 0), dims.idx3(2, 1, 1)]
    h = halo_footprint(path, dims, cost, 1, 2)
    cnt = np.bincount(h, minlength=len(dims))
    assert cnt[dims.idx3(3, 1, 0)] == 0  # an obstacle is never claimed
    # layer 0: the r = 1 box of (2,1,0) (9 cells, one obstacle) + the r = 2 via box
    # (x 0..4, y 0..3 = 20 cells, one obstacle); layer 1: the r = 1 box + the via box
    assert int((cnt[:dims.plane] > 0).sum()) == 19 and int(cnt[:dims.plane].sum()) == 8 + 19
    assert int(cnt[dims.plane:].sum()) == 9 + 20
    assert halo_footprint(path, dims, cost, 0, 0).size == 0  # both radii 0: no footprint


def _open_request(dims, pairs):
    grid = Grid.filled(dims, 1)
    nets = [NetEndpoints(f"n{i}", a, b) for i, (a, b) in enumerate(pairs)]
    return IsolatedRouteRequest(grid, nets, [IsolatedRouteWindow.full(dims)] * len(nets), [16] * (dims.w - 1),
                                [16] * (dims.h - 1), [40] * (dims.layers - 1))


def test_clearance_rounds_subtract_the_nets_own_footprint(oracle):
    """A lone net re-priced against its own path: with its own copper and
    footprint subtracted it sees the bare board and keeps its path; without
    the subtraction its own halo would push it to the other corner."""
    dims = Dims(8, 8, 1)
    req = _open_request(dims, [(dims.idx(0, 0), dims.idx(6, 6))])
    neg = SnapshotNegotiation(oracle, req, clearance=1)
    st = neg.round()
    assert st["dirty"] == 1 and st["overused_edges"] == 0 and st["next_dirty"] == 0  # converged
    first = list(neg.paths[0])
    neg.dirty = [0]  # route it once more against a snapshot that holds its own path
    neg.round()
    assert neg.paths[0] == first
    own = halo_footprint(first, dims, req.grid.cost, 1, 0)
    np.testing.assert_array_equal(neg.halo, np.bincount(own, minlength=len(dims)).astype(np.uint32))
    # the shared snapshot does carry the net's own footprint
    cell = first[len(first) // 2]
    finite = neg.snapshot[cell][neg.snapshot[cell] != COST_MAX]
    assert finite.size and (finite > 16).all()
    # ... and routed on it unsubtracted the net leaves its own path
    shared = IsolatedRouteRequest(req.grid, req.nets, req.windows, req.x_edge_costs, req.y_edge_costs,
                                  req.via_edge_costs, neg.snapshot.reshape(-1))
    assert oracle.isolated_batch(shared, retry_full=True, mode="astar")[0][0] != first


def test_clearance_rounds_route_every_net_until_no_overuse(oracle):
    """Clearance-active rounds route every net every round (no rip-up before
    pricing) while edges are overused; the halo and occupancy always equal a
    recount of the current paths; the corridor keeps both nets dirty."""
    dims, req = _corridor_request(["a", "b"])
    neg = SnapshotNegotiation(oracle, req, clearance=1, via_keepout=0)
    for _ in range(3):
        st = neg.round()
        assert st["dirty"] == 2 and st["next_dirty"] == 2 and st["overused_edges"] == 8
        np.testing.assert_array_equal(neg.present, _recount(neg))
        recount = np.zeros(len(dims), np.int64)
        for p in neg.paths:
            np.add.at(recount, halo_footprint(p, dims, req.grid.cost, 1, 0), 1)
        np.testing.assert_array_equal(neg.halo, recount.astype(np.uint32))
    wl = W.snapshot_board(w=64, h=48, layers=2, n_nets=14, median=20)
    neg = SnapshotNegotiation(oracle, wl.request(), clearance=2, via_keepout=3)
    for _ in range(6):
        st = neg.round()
        if not st["dirty"]:
            break
        assert st["dirty"] == 14
        assert st["next_dirty"] in (0, 14) and (st["next_dirty"] == 0) == (st["overused_edges"] == 0)
