"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset exists for this path, so every input is generated from a
fixed seed and every distribution choice is recorded in ``Workload.meta``.

* ``plain_board``     — 128x128x2, unit steps, via 10, ~15% blocked by
                        axis-aligned rectangles (2-12 cells a side), 64 nets on
                        free cells of random layers, whole-board windows.
* ``congestion_board`` — 512x512x4, directed planar prices
                        10 + 4*Poisson(0.3) + 3*Geom(0.2) per edge (Geom counts
                        failures before the first success, support {0,1,...}),
                        via 30, an exact 12-vertex star-radial polygon outline
                        rasterised to node and directed-edge bits with a 3-cell
                        clearance, 256 nets, windows by net_window.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .types import (
    BOARD_EDGE_NEG_X,
    BOARD_EDGE_NEG_Y,
    BOARD_EDGE_POS_X,
    BOARD_EDGE_POS_Y,
    BOARD_TRACE_NODE,
    BOARD_VIA_NODE,
    OBSTACLE,
    Dims,
    Grid,
    IsolatedRouteRequest,
    IsolatedRouteWindow,
    NetEndpoints,
)


@dataclass
class Workload:
    name: str
    grid: Grid
    nets: List[NetEndpoints]
    windows: List[IsolatedRouteWindow]
    x: np.ndarray
    y: np.ndarray
    vias: List[Optional[int]]
    directed: Optional[np.ndarray] = None
    meta: Dict = field(default_factory=dict)

    def request(self) -> IsolatedRouteRequest:
        return IsolatedRouteRequest(self.grid, self.nets, self.windows, self.x, self.y, self.vias, self.directed)

    def window_cells(self) -> int:
        return int(sum(w.cells(self.grid.dims) for w in self.windows))

    def bytes_per_cell(self) -> int:
        """Algorithmic bytes per solved cell: inputs read once + the u32 field written once."""
        b_in = 16 if self.directed is not None else 4
        if self.grid.board_constraint is not None or self.grid.via_forbidden is not None:
            b_in += 1
        return b_in + 4


def _pick_free(rng, grid: Grid, dims: Dims, legal: np.ndarray) -> int:
    free = np.flatnonzero(legal)
    return int(free[rng.integers(0, free.size)])


def _net_window(dims: Dims, net: NetEndpoints) -> IsolatedRouteWindow:
    """net_window, crates/mr-cpu/src/negotiated.rs:568-594."""
    xs = [dims.xy(c)[0] for c in [net.src, net.dst] + list(net.passable_pads)]
    ys = [dims.xy(c)[1] for c in [net.src, net.dst] + list(net.passable_pads)]
    x0, x1, y0, y1 = min(xs), max(xs), min(ys), max(ys)
    span = max(x1 - x0, y1 - y0)
    margin = max(16, (3 * span + 9) // 10)
    return IsolatedRouteWindow(max(x0 - margin, 0), max(y0 - margin, 0), min(x1 + margin, dims.w - 1),
                               min(y1 + margin, dims.h - 1))


def plain_board(seed: int = 1, w: int = 128, h: int = 128, layers: int = 2, n_nets: int = 64,
                blocked_frac: float = 0.15) -> Workload:
    rng = np.random.default_rng(seed)
    dims = Dims(w, h, layers)
    cost = np.ones((layers, h, w), dtype=np.uint32)
    while (cost == OBSTACLE).mean() < blocked_frac:
        rw, rh = int(rng.integers(2, 13)), int(rng.integers(2, 13))
        x0, y0, l = int(rng.integers(0, w - rw + 1)), int(rng.integers(0, h - rh + 1)), int(rng.integers(0, layers))
        cost[l, y0:y0 + rh, x0:x0 + rw] = OBSTACLE
    grid = Grid(dims, cost.reshape(-1))
    legal = grid.cost != OBSTACLE
    nets = []
    for i in range(n_nets):
        nets.append(NetEndpoints(f"n{i}", _pick_free(rng, grid, dims, legal), _pick_free(rng, grid, dims, legal)))
    wins = [IsolatedRouteWindow.full(dims)] * n_nets
    meta = {"workload": f"plain {w}x{h}x{layers}, {n_nets} nets", "seed": seed, "blocked_frac":
            round(float((cost == OBSTACLE).mean()), 4), "rects": "2-12 cells a side", "step": 1, "via": 10,
            "windows": "full board"}
    return Workload("plain", grid, nets, wins, np.ones(w - 1, np.uint32), np.ones(h - 1, np.uint32),
                    [10] * (layers - 1), None, meta)


def star_polygon(rng, w: int, h: int, n: int = 12) -> np.ndarray:
    """Seeded simple non-convex polygon: sorted angles, jittered radii."""
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    ang = np.sort(rng.uniform(0, 2 * np.pi, n))
    rad = rng.uniform(0.45, 0.98, n) * min(cx, cy)
    return np.stack([cx + rad * np.cos(ang), cy + rad * np.sin(ang)], axis=1)


def _inside(px, py, poly):
    inside = np.zeros(px.shape, dtype=bool)
    n = len(poly)
    for i in range(n):
        ax, ay = poly[i]
        bx, by = poly[(i + 1) % n]
        cond = (ay > py) != (by > py)
        with np.errstate(divide="ignore", invalid="ignore"):
            xint = ax + (py - ay) * (bx - ax) / (by - ay)
        inside ^= cond & (px < xint)
    return inside


def _edge_dist(px, py, poly):
    d = np.full(px.shape, np.inf)
    n = len(poly)
    for i in range(n):
        ax, ay = poly[i]
        bx, by = poly[(i + 1) % n]
        dx, dy = bx - ax, by - ay
        t = np.clip(((px - ax) * dx + (py - ay) * dy) / (dx * dx + dy * dy), 0.0, 1.0)
        d = np.minimum(d, np.hypot(px - (ax + t * dx), py - (ay + t * dy)))
    return d


def rasterise_outline(poly: np.ndarray, w: int, h: int, clearance: float = 3.0) -> np.ndarray:
    """Board mask plane with the bit layout of Grid::BOARD_* (core/src/lib.rs:411-416)
    and the edge rule of raster_mask (crates/mr-srj/src/board_outline.rs:309-352):
    a planar step is excluded in both directions when either node lies outside
    the outline or the step's midpoint is closer than `clearance` to it."""
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    inside = _inside(xs, ys, poly)
    dist = _edge_dist(xs, ys, poly)
    node_ok = inside & (dist >= clearance)
    mask = np.zeros((h, w), dtype=np.uint8)
    mask[~node_ok] |= BOARD_TRACE_NODE | BOARD_VIA_NODE
    mx, my = xs[:, :-1] + 0.5, ys[:, :-1]
    bad_h = ~inside[:, :-1] | ~inside[:, 1:] | (_edge_dist(mx, my, poly) < clearance) | ~_inside(mx, my, poly)
    mask[:, :-1][bad_h] |= BOARD_EDGE_POS_X
    mask[:, 1:][bad_h] |= BOARD_EDGE_NEG_X
    mx, my = xs[:-1, :], ys[:-1, :] + 0.5
    bad_v = ~inside[:-1, :] | ~inside[1:, :] | (_edge_dist(mx, my, poly) < clearance) | ~_inside(mx, my, poly)
    mask[:-1, :][bad_v] |= BOARD_EDGE_POS_Y
    mask[1:, :][bad_v] |= BOARD_EDGE_NEG_Y
    return mask


def congestion_board(seed: int = 2, w: int = 512, h: int = 512, layers: int = 4, n_nets: int = 256,
                     via_cost: int = 30, net_seed: Optional[int] = None) -> Workload:
    """`net_seed` (default: the board's rng stream) draws a different net set on
    the same board, e.g. one per rank."""
    rng = np.random.default_rng(seed)
    dims = Dims(w, h, layers)
    n = len(dims)
    poly = star_polygon(rng, w, h)
    plane = rasterise_outline(poly, w, h, 3.0)
    board = np.tile(plane.reshape(-1), layers)
    cost = np.ones(n, dtype=np.uint32)
    occ = rng.poisson(0.3, (n, 4))
    hist = rng.geometric(0.2, (n, 4)) - 1
    directed = (10 + 4 * occ + 3 * hist).astype(np.uint32)
    grid = Grid(dims, cost, board)
    legal = (board & BOARD_TRACE_NODE) == 0
    nrng = rng if net_seed is None else np.random.default_rng(net_seed)
    nets = []
    for i in range(n_nets):
        nets.append(NetEndpoints(f"c{i}", _pick_free(nrng, grid, dims, legal), _pick_free(nrng, grid, dims, legal)))
    wins = [_net_window(dims, nt) for nt in nets]
    meta = {"workload": f"congestion {w}x{h}x{layers}, {n_nets} nets", "seed": seed, "net_seed": net_seed,
            "edge_price": "10 + 4*Poisson(0.3) + 3*Geom(p=0.2), Geom support {0,1,...}", "via": via_cost,
            "outline": "12-vertex star-radial polygon, radii 0.45-0.98 of half-size, 3-cell clearance",
            "windows": "net_window", "board_legal_frac": round(float(legal.mean()), 4)}
    return Workload("congestion", grid, nets, wins, np.full(w - 1, 16, np.uint32), np.full(h - 1, 16, np.uint32),
                    [via_cost] * (layers - 1), directed, meta)


def scaled(wl: Workload, n_nets: int) -> Workload:
    """The same board with only the first `n_nets` nets (parity-test sizes)."""
    return Workload(wl.name, wl.grid, wl.nets[:n_nets], wl.windows[:n_nets], wl.x, wl.y, wl.vias, wl.directed,
                    dict(wl.meta, n_nets=n_nets))
