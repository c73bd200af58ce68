"""Pin the CPU oracle to the reference's own known answers (no GPU needed).

Every case in tests/golden/reference_cases.json restates a test of the
reference (its ``source`` field) and the values that test asserts.  The oracle
must reproduce all of them before any CUDA result is compared against it.
"""
import itertools

import numpy as np
import pytest

from conftest import case_grid, case_nets, load_golden
from mrcuda.types import COST_MAX, Dims, Grid, IsolatedRouteRequest, IsolatedRouteWindow, NetEndpoints

CASES = load_golden()


def _by_kind(*kinds):
    return [c for c in CASES if c["kind"] in kinds]


@pytest.mark.parametrize("case", _by_kind("lee"), ids=lambda c: c["name"])
def test_lee_known_answers(oracle, case):
    grid = case_grid(case)
    nets = case_nets(case)
    exp = case["expect"] or {}
    total = 0
    for net in nets:
        got = oracle.lee_route_one(grid, net)
        if exp.get("unrouted"):
            assert got is None
            continue
        assert got is not None, case["name"]
        path, cost = got
        total += cost
        if "cost" in exp:
            assert cost == exp["cost"]
        if "path" in exp:
            assert path == exp["path"]
        if "path_len" in exp:
            assert len(path) == exp["path_len"]
        if "field_at_dst" in exp:
            assert int(oracle.bfs_distance_field(grid, net.src)[net.dst]) == exp["field_at_dst"]
        # the Lee contract's reported cost is the sum of enter costs
        assert cost == sum(int(grid.cost[c]) if not grid.is_obstacle(c) else 1 for c in path[1:])
    if "total_cost" in exp:
        assert total == exp["total_cost"]


@pytest.mark.parametrize("case", _by_kind("lee", "field"), ids=lambda c: c["name"])
def test_sweep_field_equals_dijkstra_field(oracle, case):
    grid = case_grid(case)
    for src in range(len(grid.dims)):
        if grid.is_obstacle(src):
            continue
        a = oracle.sweep_distance_field(grid, src)
        b = oracle.bfs_distance_field(grid, src)
        assert np.array_equal(a, b), (case["name"], src)
    exp = case.get("expect") or {}
    for cell, v in (exp.get("field_values") or {}).items():
        assert int(oracle.sweep_distance_field(grid, case["nets"][0]["src"])[int(cell)]) == v


def _request(oracle, case):
    grid = case_grid(case)
    nets = case_nets(case)
    wins = case.get("windows")
    windows = ([IsolatedRouteWindow(*w) for w in wins] if wins is not None
               else [oracle.net_window(grid.dims, n) for n in nets])
    return IsolatedRouteRequest(grid, nets, windows, case["x"], case["y"], case["vias"])


@pytest.mark.parametrize("case", _by_kind("isolated", "isolated_window"), ids=lambda c: c["name"])
def test_isolated_known_answers_and_field_form_agree(oracle, case):
    req = _request(oracle, case)
    retry = case["kind"] == "isolated"
    paths, costs = oracle.isolated_batch(req, retry_full=retry, mode="astar", via_h_cost=case.get("via_h_cost"))
    # The complete-field form (h = 0, full expansion, canonical backward walk) is
    # what the GPU computes; it must select exactly the A* router's paths.
    fpaths, fcosts = oracle.isolated_batch(req, retry_full=retry, mode="field")
    assert paths == fpaths
    assert costs == fcosts
    exp = case.get("expect") or {}
    if "paths" in exp:
        assert paths == exp["paths"]
    if "search_costs" in exp:
        assert costs == exp["search_costs"]
    if "routed" in exp:
        assert [p is not None for p in paths] == exp["routed"]
    names = [n.net for n in req.nets]
    for name, p in (exp.get("paths_of") or {}).items():
        assert paths[names.index(name)] == p
    if exp.get("path_inside_window"):
        assert all(req.windows[0].contains(req.grid.dims, c) for c in paths[0])
    if "oracle_expect" in case:
        assert paths == case["oracle_expect"]["paths"]
        assert costs == case["oracle_expect"]["search_costs"]
    # Every returned path passes the router's own boundary validation.
    via_allowed = [v is not None for v in case["vias"]]
    for net, p in zip(req.nets, paths):
        if p is not None:
            assert oracle.provider_path_is_valid(req.grid, via_allowed, net, p)


@pytest.mark.parametrize("case", _by_kind("path_valid"), ids=lambda c: c["name"])
def test_provider_path_validation(oracle, case):
    grid = case_grid(case)
    net = case_nets(case)[0]
    assert oracle.provider_path_is_valid(grid, case["via_allowed"], net, case["path"]) == case["expect"]["valid"]


def test_request_edge_vectors(oracle):
    c = next(c for c in CASES if c["kind"] == "edge_vectors")
    w, h, layers = c["dims"]
    assert oracle.axis_edge_costs(c["x_lines"], w) == c["expect"]["x"]
    assert oracle.axis_edge_costs(c["y_lines"], h) == c["expect"]["y"]


def test_net_window_margin_rule(oracle):
    dims = Dims(200, 100, 2)
    # span 0 -> margin 16; clamped at the board edges
    w = oracle.net_window(dims, NetEndpoints("a", dims.idx3(5, 5, 0), dims.idx3(5, 5, 1)))
    assert (w.x0, w.y0, w.x1, w.y1) == (0, 0, 21, 21)
    # bbox x 40..150 (the pad widens it), span 110 -> margin ceil(33) = 33
    n = NetEndpoints("b", dims.idx3(50, 40, 0), dims.idx3(150, 60, 1), passable_pads=[dims.idx3(40, 45, 0)])
    w = oracle.net_window(dims, n)
    assert (w.x0, w.y0, w.x1, w.y1) == (40 - 33, 40 - 33, 150 + 33, 60 + 33)


def test_exhaustive_3x3_masks_sweep_and_walk_match_lee(oracle):
    """crates/mr-cpu/src/sweep.rs:301-330, every obstacle mask of a 3x3 grid."""
    dims = Dims(3, 3)
    for mask in range(1 << 9):
        cost = np.ones(9, dtype=np.uint32)
        for c in range(9):
            if mask & (1 << c):
                cost[c] = COST_MAX
        grid = Grid(dims, cost)
        for src in range(9):
            if grid.is_obstacle(src):
                continue
            sweep = oracle.sweep_distance_field(grid, src)
            assert np.array_equal(sweep, oracle.bfs_distance_field(grid, src))
            for dst in range(9):
                if grid.is_obstacle(dst):
                    continue
                got = oracle.path_from_field(grid, sweep, src, dst)
                lee = oracle.lee_route_one(grid, NetEndpoints("n", src, dst))
                assert got == (lee[0] if lee else None), (mask, src, dst)


def test_astar_equals_field_walk_on_seeded_weighted_multilayer_grids(oracle):
    """The A* router's canonical path equals the complete-field backward walk,
    across zero costs, obstacles, own pads, board masks and restricted vias."""
    rng = np.random.default_rng(7)
    for trial in range(40):
        w, h, layers = int(rng.integers(2, 9)), int(rng.integers(2, 8)), int(rng.integers(1, 4))
        dims = Dims(w, h, layers)
        n = len(dims)
        cost = rng.integers(0, 6, n).astype(np.uint32)
        cost[rng.random(n) < 0.2] = COST_MAX
        board = None
        if trial % 3 == 0:
            board = (rng.random(n) < 0.3).astype(np.uint8) * rng.integers(0, 64, n).astype(np.uint8)
            board &= ~np.uint8(1)  # keep nodes legal, exercise edge and via bits
        vf = (rng.random(n) < 0.3).astype(np.uint8) if trial % 4 == 1 else None
        grid = Grid(dims, cost, board, vf)
        x = rng.integers(0, 40, max(w - 1, 0)).tolist()
        y = rng.integers(0, 40, max(h - 1, 0)).tolist()
        vias = [None if rng.random() < 0.3 else int(rng.integers(0, 50)) for _ in range(layers - 1)]
        nets = []
        for i in range(6):
            src, dst = int(rng.integers(0, n)), int(rng.integers(0, n))
            pads = [c for c in (src, dst) if grid.is_obstacle(c)]
            vpads = [c for c in pads if rng.random() < 0.5]
            nets.append(NetEndpoints(f"t{trial}-{i}", src, dst, sorted(set(pads)), sorted(set(vpads))))
        wins = [IsolatedRouteWindow.full(dims) if i % 2 else oracle.net_window(dims, nn) for i, nn in enumerate(nets)]
        req = IsolatedRouteRequest(grid, nets, wins, x, y, vias)
        a = oracle.isolated_batch(req, mode="astar")
        b = oracle.isolated_batch(req, mode="field")
        assert a == b, trial


def test_directed_superset_equals_axis_form_when_tables_match(oracle):
    """Per-edge base prices that repeat the axis gap prices give identical paths."""
    rng = np.random.default_rng(3)
    dims = Dims(11, 9, 3)
    cost = rng.integers(1, 5, len(dims)).astype(np.uint32)
    cost[rng.random(len(dims)) < 0.15] = COST_MAX
    grid = Grid(dims, cost)
    x = rng.integers(1, 30, dims.w - 1)
    y = rng.integers(1, 30, dims.h - 1)
    d = np.zeros((len(dims), 4), dtype=np.uint32)
    for c in range(len(dims)):
        cx, cy, _ = dims.xyz(c)
        d[c] = [y[cy - 1] if cy > 0 else 0, x[cx - 1] if cx > 0 else 0, x[cx] if cx + 1 < dims.w else 0,
                y[cy] if cy + 1 < dims.h else 0]
    nets = [NetEndpoints(f"n{i}", int(s), int(t)) for i, (s, t) in
            enumerate(rng.integers(0, len(dims), (10, 2)))]
    nets = [n for n in nets if not grid.is_obstacle(n.src) and not grid.is_obstacle(n.dst)]
    wins = [IsolatedRouteWindow.full(dims)] * len(nets)
    plain = oracle.isolated_batch(IsolatedRouteRequest(grid, nets, wins, x, y, [20, None]), mode="field")
    directed = oracle.isolated_batch(IsolatedRouteRequest(grid, nets, wins, x, y, [20, None], d), mode="field")
    assert plain == directed
