"""The reference's isolated-provider contract, checked against libmr_cuda.so.

The reference pins the seam between NegotiatedRouter and an accelerated
isolated-route provider with its own tests: reachable, unreachable and
zero-hop nets (crates/mr-cpu/src/negotiated.rs:4451-4483), whole-batch
all-or-error behaviour (:4486-4516), the exact request edge vectors
(:4659-4705), the adapter's window-then-full retry that keeps results aligned
with the nets (crates/mr-cli/src/lib.rs:2204-2264, :2266-2300) and, where the
Metal backend had to fail closed, static via masks and board masks
(:2302-2385).  Those tests drive Rust types this image cannot build, so the
contract they pin is exercised here through the C ABI (ctypes), against the
CPU oracle, on both relax schedules.
"""
import ctypes as C

import numpy as np
import pytest

import mrcuda
from mrcuda import api
from mrcuda.types import COST_MAX, Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[1, 2], ids=["cta-tiles", "warp-tiles"])
def engine(request):
    e = mrcuda.Engine(0)
    e.set_schedule(request.param)
    yield e
    e.close()


def _windows(oracle, grid, nets):
    return [oracle.net_window(grid.dims, n) for n in nets]


def _check_against_oracle(oracle, engine, req, retry=True):
    got = engine.route_isolated_batch(req, retry_full=retry)
    exp_paths, exp_costs = oracle.isolated_batch(req, retry_full=retry, mode="field")
    assert got.paths == exp_paths
    assert got.search_costs == exp_costs
    via_allowed = [v is not None for v in req.via_edge_costs]
    for net, p in zip(req.nets, got.paths):
        if p is not None:
            assert oracle.provider_path_is_valid(req.grid, via_allowed, net, p)
    return got


def test_reachable_unreachable_and_zero_hop_nets(engine, oracle):
    """negotiated.rs:4451-4483: an enclosed target is unreachable (None), a
    zero-length net returns [src], and the open net its canonical path."""
    dims = Dims(5, 5)
    grid = Grid.filled(dims, 1)
    for x, y in [(2, 1), (1, 2), (3, 2), (2, 3)]:
        grid.set(dims.idx(x, y), COST_MAX)
    nets = [NetEndpoints("open", dims.idx(0, 4), dims.idx(4, 4)),
            NetEndpoints("blocked", dims.idx(0, 0), dims.idx(2, 2)),
            NetEndpoints("zero", dims.idx(4, 0), dims.idx(4, 0))]
    x, y = oracle.axis_edge_costs([], 5), oracle.axis_edge_costs([], 5)
    req = IsolatedRouteRequest(grid, nets, _windows(oracle, grid, nets), x, y, [])
    got = _check_against_oracle(oracle, engine, req)
    assert got.paths[1] is None and got.paths[2] == [nets[2].src]
    assert got.paths[0][0] == nets[0].src and got.paths[0][-1] == nets[0].dst
    # the seam itself: one aligned Option per net
    prov = mrcuda.CudaIsolatedProvider(engine)
    assert prov.route_isolated_batch(req) == got.paths


def test_errors_are_all_or_nothing(engine):
    """negotiated.rs:4486-4516: any failure rejects the whole batch.  A batch
    with one bad net returns an error status and no result object at all."""
    lib = engine.lib
    dims = Dims(5, 5)
    grid = Grid.filled(dims, 1)
    grid.set(dims.idx(2, 2), COST_MAX)
    nets = [NetEndpoints("ok", dims.idx(0, 0), dims.idx(4, 0)),
            NetEndpoints("foreign-obstacle", dims.idx(0, 4), dims.idx(2, 2))]
    req = IsolatedRouteRequest(grid, nets, [IsolatedRouteWindow.full(dims)] * 2, [16] * 4, [16] * 4, [])
    m = api._Marshal()
    r = engine._request(m, req)
    res = C.c_void_p()
    st = lib.mrc_route_isolated_batch(engine.ctx, C.byref(r), api.MRC_FLAG_RETRY_FULL, C.byref(res))
    assert st == mrcuda.InvalidEndpoint.status  # MRC_ERR_INVALID_ENDPOINT
    assert not res.value, "no partial output on error"
    with pytest.raises(mrcuda.InvalidEndpoint):
        mrcuda.CudaIsolatedProvider(engine).route_isolated_batch(req)
    # the engine keeps serving after the refusal
    ok = IsolatedRouteRequest(grid, nets[:1], [IsolatedRouteWindow.full(dims)], [16] * 4, [16] * 4, [])
    assert engine.route_isolated_batch(ok).paths[0] is not None


def test_request_uses_the_exact_short_coordinate_and_via_vectors(engine, oracle):
    """negotiated.rs:4659-4705: a 4x3x3 board with one x coordinate line gives
    x = [144, 16, 16], y = [16, 16] and vias [Some(7), None]; the engine
    routes that request exactly as the CPU does."""
    dims = Dims(4, 3, 3)
    grid = Grid.filled(dims, 1)
    x, y = oracle.axis_edge_costs([10.0], 4), oracle.axis_edge_costs([], 3)
    assert list(x) == [144, 16, 16] and list(y) == [16, 16]
    nets = [NetEndpoints("n", dims.idx3(0, 0, 0), dims.idx3(3, 2, 0)),
            NetEndpoints("up", dims.idx3(1, 1, 0), dims.idx3(1, 1, 1)),
            NetEndpoints("forbidden-step", dims.idx3(1, 1, 1), dims.idx3(1, 1, 2))]
    req = IsolatedRouteRequest(grid, nets, [IsolatedRouteWindow.full(dims)] * 3, x, y, [7, None])
    got = _check_against_oracle(oracle, engine, req)
    assert got.paths[1] == [nets[1].src, nets[1].dst] and got.search_costs[1] == 7
    assert got.paths[2] is None  # the 1 <-> 2 transition is None: no via reaches layer 2


def test_window_failures_retry_on_the_full_board_and_stay_aligned(engine, oracle):
    """cli/src/lib.rs:2204-2264: only the nets unreachable in their windows are
    solved again on the whole board, and the answers come back in the nets'
    order (the middle net keeps its window path)."""
    dims = Dims(20, 9)
    grid = Grid.filled(dims, 1)
    for yy in range(0, 8):  # a wall with one gap at the bottom row
        grid.set(dims.idx(10, yy), COST_MAX)
    nets = [NetEndpoints("n0", dims.idx(8, 1), dims.idx(12, 1)),
            NetEndpoints("n1", dims.idx(1, 4), dims.idx(5, 4)),
            NetEndpoints("n2", dims.idx(9, 3), dims.idx(11, 3))]
    wins = [IsolatedRouteWindow(7, 0, 13, 4), IsolatedRouteWindow(0, 2, 6, 6), IsolatedRouteWindow(8, 2, 12, 5)]
    req = IsolatedRouteRequest(grid, nets, wins, [16] * 19, [16] * 8, [])
    window_only = _check_against_oracle(oracle, engine, req, retry=False)
    assert window_only.paths[0] is None and window_only.paths[2] is None
    assert window_only.paths[1] is not None
    got = _check_against_oracle(oracle, engine, req, retry=True)
    assert got.retried == 2
    assert got.paths[1] == window_only.paths[1]
    assert all(p is not None for p in got.paths)
    assert all(dims.idx(10, 8) in p for p in (got.paths[0], got.paths[2]))  # through the gap


def _ragged_adapter_case(oracle):
    """The 9x7x3 weighted board of cli/src/lib.rs:2302-2330: uneven coordinate
    lines, a zero-cost and a weight-7 cell, four obstacles, two of them the
    endpoints of a net that owns them, a zero-length net and vias of 37."""
    dims = Dims(9, 7, 3)
    x = oracle.axis_edge_costs([0.0, 0.2, 0.7, 1.9, 2.0, 4.5, 4.7, 8.0, 8.1], 9)
    y = oracle.axis_edge_costs([0.0, 0.1, 1.0, 1.0, 2.7, 6.0, 6.2], 7)
    grid = Grid.filled(dims, 1)
    grid.set(dims.idx3(2, 3, 0), 0)
    grid.set(dims.idx3(3, 3, 1), 7)
    for xx, yy, ll in [(0, 0, 0), (8, 0, 2), (4, 3, 0), (4, 3, 1)]:
        grid.set(dims.idx3(xx, yy, ll), COST_MAX)
    nets = [NetEndpoints("weighted", dims.idx3(0, 3, 0), dims.idx3(8, 3, 2)),
            NetEndpoints("own-pads", dims.idx3(0, 0, 0), dims.idx3(8, 0, 2),
                         [dims.idx3(0, 0, 0), dims.idx3(8, 0, 2)]),
            NetEndpoints("zero-length", dims.idx3(2, 3, 0), dims.idx3(2, 3, 0))]
    return dims, grid, nets, x, y, [37, 37]


def test_static_via_mask_and_board_mask_are_routed_exactly(engine, oracle):
    """cli/src/lib.rs:2302-2385: where the Metal backend had to fail closed (a
    selected static via mask, an exact board mask with a directed edge bit) and
    hand the batch back to the CPU, this engine carries both masks and returns
    the CPU's exact answer itself."""
    dims, grid, nets, x, y, vias = _ragged_adapter_case(oracle)
    plain = IsolatedRouteRequest(grid, nets, _windows(oracle, grid, nets), x, y, vias)
    got_plain = _check_against_oracle(oracle, engine, plain)
    assert got_plain.paths[2] == [nets[2].src]
    masked = Grid(dims, grid.cost.copy(), None, np.zeros(len(dims), np.uint8))
    _check_against_oracle(oracle, engine, IsolatedRouteRequest(masked, nets, plain.windows, x, y, vias))
    board = np.zeros(len(dims), np.uint8)
    board[dims.idx3(1, 1, 0)] |= 1 << 4  # BOARD_EDGE_POS_X
    outlined = Grid(dims, grid.cost.copy(), board, None)
    _check_against_oracle(oracle, engine, IsolatedRouteRequest(outlined, nets, plain.windows, x, y, vias))
    # and a static via mask that really forbids vias, with one exempt pad
    vf = np.ones(len(dims), np.uint8)
    exempt = [NetEndpoints(n.net, n.src, n.dst, n.passable_pads, n.passable_pads) for n in nets]
    _check_against_oracle(oracle, engine, IsolatedRouteRequest(Grid(dims, grid.cost.copy(), None, vf), exempt,
                                                               plain.windows, x, y, vias))
