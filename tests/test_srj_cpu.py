"""The SimpleRouteJson input side on the CPU: the synthetic problem generator,
the resolution policy, rasterisation to a routing request and the solution
soup (routed here by the CPU oracle; the GPU test of /solve routes them on the
device)."""
import math

import numpy as np
import pytest

from mrcuda import srj
from mrcuda.types import OBSTACLE


def test_generated_problem_is_deterministic_and_well_formed():
    """crates/mr-cli/src/bench.rs:259-270: 60 connections, 8 obstacles, the same
    first endpoint from the same seed."""
    a = srj.generate_problem(7, 30.0, 8, 60)
    b = srj.generate_problem(7, 30.0, 8, 60)
    assert len(a["connections"]) == 60 and len(a["obstacles"]) == 8
    assert a == b
    assert srj.generate_problem(8, 30.0, 8, 60) != a
    size, margin = 30.0, max(30.0 / 64.0, 0.5)
    for ob in a["obstacles"]:
        assert 0.15 * size <= ob["center"]["x"] < 0.85 * size
        assert 0.04 * size <= ob["width"] < 0.16 * size
    for con in a["connections"]:
        for p in con["pointsToConnect"]:
            clear = all(abs(p["x"] - o["center"]["x"]) > o["width"] / 2 + margin or
                        abs(p["y"] - o["center"]["y"]) > o["height"] / 2 + margin for o in a["obstacles"])
            assert clear or p["x"] < 0.04 * size  # else the obstacle-free edge band


def test_lcg_stream():
    """The generator's LCG, stepped by hand for the first outputs of seed 0."""
    g = srj._Lcg(0)
    s = 3037000493
    for _ in range(3):
        s = (s * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        assert g.next_u64() == s >> 16


def test_resolution_policy():
    base = {"bounds": {"minX": 0.0, "maxX": 100.0, "minY": 0.0, "maxY": 40.0}, "layerCount": 1}
    assert srj.choose_resolution(base) == pytest.approx(0.5)
    assert srj.choose_resolution(base, 0.25) == 0.25
    assert srj.choose_resolution(base, -1.0) == pytest.approx(0.5)
    assert srj.choose_resolution(dict(base, minTraceWidth=0.15)) == pytest.approx(0.3)
    small = {"bounds": {"minX": 0.0, "maxX": 5.0, "minY": 0.0, "maxY": 5.0}, "layerCount": 1}
    assert srj.choose_resolution(small) == srj.MIN_RESOLUTION
    assert srj.edge_cost(0.5) == 8 and srj.edge_cost(0.03125) == 1 and srj.edge_cost(0.0) == 0


def test_rasterize_blocks_obstacles_and_snaps_points():
    prob_json = {
        "layerCount": 2,
        "bounds": {"minX": 0.0, "maxX": 10.0, "minY": 0.0, "maxY": 5.0},
        "obstacles": [{"type": "rect", "center": {"x": 5.0, "y": 2.5}, "width": 2.0, "height": 2.0,
                       "layers": ["top"]}],
        "connections": [{"name": "a", "pointsToConnect": [{"x": 0.26, "y": 0.24}, {"x": 9.74, "y": 4.9}]},
                        {"name": "m", "pointsToConnect": [{"x": 1.0, "y": 1.0}, {"x": 2.0, "y": 1.0},
                                                          {"x": 2.0, "y": 3.0, "layer": "bottom"}]}],
    }
    p = srj.rasterize(prob_json, 0.5)
    dims = p.request.grid.dims
    assert (dims.w, dims.h, dims.layers) == (21, 11, 2)
    cost = p.request.grid.cost.reshape(2, 11, 21)
    assert (cost[0, 3:8, 8:13] == OBSTACLE).all() and (cost[1] != OBSTACLE).all()
    assert cost[0, 2, 8] != OBSTACLE
    nets = p.request.nets
    assert [n.net for n in nets] == ["a", "m#seg0", "m#seg1"]
    # nearest line, ties to the lower index: x 0.26 -> 0.5, y 0.24 -> 0.0
    assert dims.xyz(nets[0].src) == (1, 0, 0) and dims.xyz(nets[0].dst) == (19, 10, 0)
    assert dims.xyz(nets[2].dst) == (4, 6, 1)
    assert list(p.request.x_edge_costs) == [8] * 20 and p.request.via_edge_costs == [srj.VIA_STEP_COST]


def test_soup_of_oracle_paths(oracle):
    prob_json = srj.generate_problem(3, 20.0, 5, 12)
    p = srj.rasterize(prob_json, srj.choose_resolution(prob_json, 0.5), layers=2)
    paths, costs = oracle.isolated_batch(p.request, retry_full=True, mode="astar")
    soup = srj.solution_soup(p, paths)
    assert len(soup) == sum(1 for q in paths if q and len(q) > 1)
    for tr, path in zip(soup, [q for q in paths if q and len(q) > 1]):
        assert tr["type"] == "pcb_trace"
        r = tr["route"]
        dims = p.request.grid.dims
        (sx, sy, _), (dx, dy, _) = dims.xyz(path[0]), dims.xyz(path[-1])
        assert (r[0]["x"], r[0]["y"]) == (p.x_lines[sx], p.y_lines[sy])
        assert (r[-1]["x"], r[-1]["y"]) == (p.x_lines[dx], p.y_lines[dy])
        wires = [q for q in r if q["route_type"] == "wire"]
        for u, v in zip(wires, wires[1:]):  # every wire segment is axis-aligned (or a via's two ends)
            assert u["x"] == v["x"] or u["y"] == v["y"]
        assert sum(q["route_type"] == "via" for q in r) == sum(
            dims.xyz(a)[2] != dims.xyz(b)[2] for a, b in zip(path, path[1:]))
