"""The SimpleRouteJson input side of the path: problems in, routing grids out,
paths back to the tscircuit solution soup.

* ``generate_problem`` — the deterministic synthetic problem generator of the
  reference's CPU bench (crates/mr-cli/src/bench.rs:88-176): the same LCG
  stream, rectangles with centres in [0.15, 0.85]·size and sides in
  [0.04, 0.16]·size, endpoints drawn clear of every obstacle by a margin of
  max(size/64, 0.5) (32 tries, then the obstacle-free edge band), one layer.
* ``choose_resolution`` — the server's cell-size policy
  (crates/mr-server/src/lib.rs:173-203): a caller override, else the longer
  bounds span / 200 floored at 0.1, capped at two minimum trace widths.
* ``rasterize`` — a uniform-pitch restatement of the reference rasteriser
  (crates/mr-srj/src/lib.rs:1364-1794).  Grid lines run at min + k·resolution on
  both axes (the reference draws non-uniform Hanan lines through every pad and
  obstacle edge; on the generator's problems, whose points are continuous, the
  uniform lattice is the resolution the reference falls back to for its fill
  channels).  An obstacle blocks the nodes inside its rectangle grown by the
  clearance halo on each of its layers (every layer when it names none); a
  polygon ``outline`` becomes node and directed-edge board bits by the rule of
  raster_mask (crates/mr-srj/src/board_outline.rs:309-352), replicated on every
  layer (lib.rs:1764-1794).  Connection points snap to the nearest line
  (Mapping::point_to_xy, ties to the lower index); a point that lands on an
  obstacle becomes one of its own net's passable pads.  A connection with more
  than two points is split into consecutive two-point segments named
  ``name#seg<k>``.  Edge prices come from the lines exactly as the router
  derives them (axis_gap_cost, crates/mr-cpu/src/negotiated.rs:1197-1201, with
  edge_cost, dijkstra.rs:36-52) and vias from ViaModel::through_hole.
* ``solution_soup`` — one ``pcb_trace`` per routed net: wire points at the ends
  and every change of direction, a via point at every layer change
  (RoutePoint / PcbTrace, crates/mr-srj/src/lib.rs:2231-2260).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .types import OBSTACLE, Dims, Grid, IsolatedRouteRequest, NetEndpoints
from .workloads import _net_window, rasterise_outline

TARGET_CELLS_PER_AXIS = 200.0  # crates/mr-server/src/lib.rs:58
MIN_RESOLUTION = 0.1           # :62
DEFAULT_TRACE_WIDTH = 0.15     # :65
COST_SCALE = 16.0              # crates/mr-cpu/src/dijkstra.rs:36
VIA_STEP_COST = 160            # ViaModel::DEFAULT_STEP_COST (crates/mr-core/src/lib.rs), through_hole's

_M64 = (1 << 64) - 1


class _Lcg:
    """The generator's LCG: state' = state * 6364136223846793005 +
    1442695040888963407 (mod 2^64), output state' >> 16."""

    def __init__(self, seed: int):
        self.s = (seed * 2862933555777941757 + 3037000493) & _M64

    def next_u64(self) -> int:
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & _M64
        return self.s >> 16

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (self.next_u64() % 100_000) / 100_000.0 * (hi - lo)


def generate_problem(seed: int, size: float, n_obstacles: int, n_nets: int) -> dict:
    """A deterministic SimpleRouteJson problem (the JSON object, camelCase keys)."""
    rng = _Lcg(seed)
    rects = []
    for _ in range(n_obstacles):
        cx = rng.uniform(0.15 * size, 0.85 * size)
        cy = rng.uniform(0.15 * size, 0.85 * size)
        w = rng.uniform(0.04 * size, 0.16 * size)
        h = rng.uniform(0.04 * size, 0.16 * size)
        rects.append((cx, cy, w / 2.0, h / 2.0))
    margin = max(size / 64.0, 0.5)

    def in_obstacle(x, y):
        return any(abs(x - cx) <= hw + margin and abs(y - cy) <= hh + margin for cx, cy, hw, hh in rects)

    def sample_point():
        for _ in range(32):
            x = rng.uniform(0.02 * size, 0.98 * size)
            y = rng.uniform(0.02 * size, 0.98 * size)
            if not in_obstacle(x, y):
                return x, y
        return rng.uniform(0.01 * size, 0.04 * size), rng.uniform(0.01 * size, 0.96 * size)

    connections = []
    for i in range(n_nets):
        ax, ay = sample_point()
        bx, by = sample_point()
        connections.append({"name": f"n{i}", "pointsToConnect": [{"x": ax, "y": ay}, {"x": bx, "y": by}]})
    return {
        "layerCount": 1,
        "bounds": {"minX": 0.0, "maxX": size, "minY": 0.0, "maxY": size},
        "obstacles": [{"type": "rect", "center": {"x": cx, "y": cy}, "width": hw * 2.0, "height": hh * 2.0}
                      for cx, cy, hw, hh in rects],
        "connections": connections,
    }


def choose_resolution(srj: dict, override: Optional[float] = None) -> float:
    if override is not None and math.isfinite(override) and override > 0.0:
        return float(override)
    b = srj["bounds"]
    span = max(max(b["maxX"] - b["minX"], 0.0), max(b["maxY"] - b["minY"], 0.0))
    if span <= 0.0:
        return MIN_RESOLUTION
    res = max(span / TARGET_CELLS_PER_AXIS, MIN_RESOLUTION)
    w = srj.get("minTraceWidth")
    if w is not None and math.isfinite(w) and w > 0.0:
        res = min(res, max(w * 2.0, MIN_RESOLUTION))
    return res


def edge_cost(length: float) -> int:
    """round(length * 16), half away from zero, saturating (dijkstra.rs:36-52)."""
    scaled = math.floor(abs(length) * COST_SCALE + 0.5) if length >= 0 else 0
    if not math.isfinite(scaled) or scaled <= 0:
        return 0
    return min(int(scaled), OBSTACLE)


def layer_index(name: str, layers: int) -> int:
    """LayerMap::standard: "top" = 0, "bottom" = the last layer, "innerN" = N."""
    n = name.lower()
    if n in ("top", "f.cu", "front"):
        return 0
    if n in ("bottom", "b.cu", "back"):
        return layers - 1
    if n.startswith("inner"):
        try:
            return min(max(int(n[5:]), 1), layers - 1)
        except ValueError:
            return 0
    return 0


@dataclass
class RasterizedProblem:
    """A routing request plus the mapping back to continuous coordinates."""

    request: IsolatedRouteRequest
    x_lines: np.ndarray
    y_lines: np.ndarray
    layer_names: List[str]
    trace_width: float
    connection_of: List[str] = field(default_factory=list)  # the SRJ connection of every net


def _nearest(lines: np.ndarray, v: float) -> int:
    """Index of the nearest line, ties to the lower index, clamped."""
    i = int(np.searchsorted(lines, v))
    if i <= 0:
        return 0
    if i >= len(lines):
        return len(lines) - 1
    return i - 1 if (v - lines[i - 1]) <= (lines[i] - v) else i


def rasterize(srj: dict, resolution: float, layers: int = 0, clearance_cells: int = 0) -> RasterizedProblem:
    b = srj["bounds"]
    L = max(int(srj.get("layerCount", 1) or 1), int(layers), 1)
    nx = max(int(math.floor((b["maxX"] - b["minX"]) / resolution + 1e-9)) + 1, 1)
    ny = max(int(math.floor((b["maxY"] - b["minY"]) / resolution + 1e-9)) + 1, 1)
    x_lines = b["minX"] + resolution * np.arange(nx, dtype=np.float64)
    y_lines = b["minY"] + resolution * np.arange(ny, dtype=np.float64)
    dims = Dims(nx, ny, L)
    cost = np.ones((L, ny, nx), dtype=np.uint32)
    grow = clearance_cells * resolution
    for ob in srj.get("obstacles", []):
        cx, cy = ob["center"]["x"], ob["center"]["y"]
        hw, hh = ob["width"] / 2.0 + grow, ob["height"] / 2.0 + grow
        xs = np.flatnonzero((x_lines >= cx - hw) & (x_lines <= cx + hw))
        ys = np.flatnonzero((y_lines >= cy - hh) & (y_lines <= cy + hh))
        if xs.size == 0 or ys.size == 0:
            continue
        names = ob.get("layers") or []
        lays = sorted({layer_index(n, L) for n in names}) if names else range(L)
        for l in lays:
            cost[l, ys[0]:ys[-1] + 1, xs[0]:xs[-1] + 1] = OBSTACLE
    board = None
    outline = srj.get("outline")
    if outline:
        poly = np.array([[(p["x"] - b["minX"]) / resolution, (p["y"] - b["minY"]) / resolution] for p in outline])
        plane = rasterise_outline(poly, nx, ny, clearance=float(clearance_cells))
        board = np.tile(plane.reshape(-1), L)
    cost = cost.reshape(-1)
    nets, names = [], []
    for con in srj.get("connections", []):
        pts = con.get("pointsToConnect", [])
        cells = []
        for p in pts:
            l = layer_index(p["layer"], L) if "layer" in p else 0
            cells.append(dims.idx3(_nearest(x_lines, p["x"]), _nearest(y_lines, p["y"]), l))
        segs = list(zip(cells[:-1], cells[1:]))
        for k, (a, c) in enumerate(segs):
            nm = con["name"] if len(segs) == 1 else f"{con['name']}#seg{k}"
            pads = sorted({q for q in (a, c) if cost[q] == OBSTACLE})
            nets.append(NetEndpoints(nm, a, c, pads))
            names.append(con["name"])
    grid = Grid(dims, cost, board)
    x = np.array([edge_cost(x_lines[k + 1] - x_lines[k]) for k in range(nx - 1)], dtype=np.uint32)
    y = np.array([edge_cost(y_lines[k + 1] - y_lines[k]) for k in range(ny - 1)], dtype=np.uint32)
    vias = [VIA_STEP_COST] * (L - 1)
    windows = [_net_window(dims, n) for n in nets]
    width = srj.get("minTraceWidth") or DEFAULT_TRACE_WIDTH
    layer_names = ["top"] + [f"inner{k}" for k in range(1, L - 1)] + (["bottom"] if L > 1 else [])
    return RasterizedProblem(IsolatedRouteRequest(grid, nets, windows, x, y, vias), x_lines, y_lines, layer_names,
                             float(width), names)


def solution_soup(prob: RasterizedProblem, paths: Sequence[Optional[Sequence[int]]]) -> List[dict]:
    """``pcb_trace`` objects of the routed nets (unrouted nets emit nothing)."""
    dims = prob.request.grid.dims
    out = []
    for path in paths:
        if not path or len(path) < 2:
            continue
        route = []
        pts = [dims.xyz(c) for c in path]
        for k, (x, y, l) in enumerate(pts):
            wx, wy = float(prob.x_lines[x]), float(prob.y_lines[y])
            if k > 0 and pts[k - 1][2] != l:  # a layer change: a via between the two cells
                route.append({"route_type": "via", "x": wx, "y": wy, "from_layer": prob.layer_names[pts[k - 1][2]],
                              "to_layer": prob.layer_names[l]})
                route.append({"route_type": "wire", "x": wx, "y": wy, "width": prob.trace_width,
                              "layer": prob.layer_names[l]})
                continue
            keep = k == 0 or k == len(pts) - 1
            if not keep:
                px, py, pl = pts[k - 1]
                qx, qy, ql = pts[k + 1]
                keep = ql != l or (x - px, y - py) != (qx - x, qy - y)  # a turn or a via next
            if keep:
                route.append({"route_type": "wire", "x": wx, "y": wy, "width": prob.trace_width,
                              "layer": prob.layer_names[l]})
        out.append({"type": "pcb_trace", "route": route})
    return out
