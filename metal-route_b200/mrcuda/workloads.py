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
* ``uneven_instances`` — 4096 independent one-net instances whose bounding
                        boxes have log-normal sides (median 96, sigma 0.5,
                        clamped 16-1024), 2-8 layers, pad clusters with keepout
                        halos and courtyard edge bits, unit steps, via 10.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

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


def pin_boards(engine, boards: Sequence["Workload"]) -> None:
    """Moves every workload's board arrays (cost, masks, directed prices) into
    one page-locked block of `engine` (64-byte aligned views), in place."""
    arrays = []
    for wl in boards:
        g = wl.grid
        arrays += [g.cost, g.board_constraint, g.via_forbidden, wl.directed]
    offs, tot = [], 0
    for a in arrays:
        offs.append(tot)
        tot += 0 if a is None else (a.nbytes + 63) & ~63
    blk = engine.pinned_empty(max(tot, 1), np.uint8)

    def view(a, o):
        if a is None:
            return None
        v = blk[o:o + a.nbytes].view(a.dtype).reshape(a.shape)
        v[...] = a
        return v

    for k, wl in enumerate(boards):
        c, b, vf, d = (view(arrays[4 * k + i], offs[4 * k + i]) for i in range(4))
        wl.grid = Grid(wl.grid.dims, c, b, vf)
        wl.directed = d


_FREE_CACHE: Dict[int, tuple] = {}


def _pick_free(rng, grid: Grid, dims: Dims, legal: np.ndarray) -> int:
    hit = _FREE_CACHE.get(id(legal))
    if hit is None or hit[0] is not legal:
        _FREE_CACHE.clear()
        hit = (legal, np.flatnonzero(legal))
        _FREE_CACHE[id(legal)] = hit
    free = hit[1]
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


@dataclass
class InstanceSet:
    """Many independent instances (each its own board and nets) solved together."""

    name: str
    instances: List[Workload]
    meta: Dict = field(default_factory=dict)

    def requests(self) -> List[IsolatedRouteRequest]:
        return [w.request() for w in self.instances]

    @property
    def n_nets(self) -> int:
        return sum(len(w.nets) for w in self.instances)

    def window_cells(self) -> int:
        return sum(w.window_cells() for w in self.instances)

    def algorithmic_bytes(self) -> int:
        """Sum over instances of window cells x bytes per cell (paths excluded)."""
        return sum(w.window_cells() * w.bytes_per_cell() for w in self.instances)


def _footprint(rng, w: int, h: int) -> Optional[tuple]:
    """One pad cluster: 4-40 pads in one or two rows on a 2-5 cell pitch."""
    n_pads = int(rng.integers(4, 41))
    pitch = int(rng.integers(2, 6))
    halo = int(rng.integers(1, 3))
    rows = 1 if n_pads < 8 or rng.random() < 0.5 else 2
    gap = 3 * pitch
    per_row = (n_pads + rows - 1) // rows
    vertical = bool(rng.random() < 0.5)
    along, across = (h, w) if vertical else (w, h)
    room = along - 2 * halo - 2
    per_row = max(1, min(per_row, room // pitch + 1))
    span_along = (per_row - 1) * pitch
    span_across = (rows - 1) * gap
    if span_along + 2 * halo + 2 > along or span_across + 2 * halo + 2 > across:
        rows, span_across = 1, 0
        if span_along + 2 * halo + 2 > along:
            return None
    a0 = int(rng.integers(halo + 1, along - halo - span_along))
    c0 = int(rng.integers(halo + 1, across - halo - span_across))
    pads = []
    for r in range(rows):
        for i in range(per_row):
            a, c = a0 + i * pitch, c0 + r * gap
            pads.append((c, a) if vertical else (a, c))
    return pads, halo


def uneven_instances(seed: int = 3, n_instances: int = 4096, median: float = 96.0, sigma: float = 0.5,
                     lo: int = 16, hi: int = 1024, min_layers: int = 2, max_layers: int = 8) -> InstanceSet:
    """Independent two-pin instances of uneven size, one net each; an instance is
    its net's bounding box, solved whole (window = the instance).

    Box side ~ LogNormal(ln median, sigma) clamped to [lo, hi], per axis; layers
    uniform in [min_layers, max_layers]; unit enter weights, unit x/y steps, via
    10.  Two to four pad clusters (4-40 pads, one or two rows, 2-5 cell pitch) on
    the top or bottom layer: pads and a 1-2 cell keepout halo are obstacles;
    the cluster's courtyard (its bounding box grown by the halo + 1) refuses
    planar steps entering it on the pad layer (incoming directed-edge bits), so
    a trace reaches a pad through its own halo or a via.  The net joins a pad of
    the first cluster to a pad of the second; its passable pads are both pads
    and their halo cells."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_instances):
        w = int(np.clip(round(median * np.exp(sigma * rng.standard_normal())), lo, hi))
        h = int(np.clip(round(median * np.exp(sigma * rng.standard_normal())), lo, hi))
        layers = int(rng.integers(min_layers, max_layers + 1))
        dims = Dims(w, h, layers)
        cost = np.ones((layers, h, w), dtype=np.uint32)
        board = np.zeros((layers, h, w), dtype=np.uint8)
        clusters = []
        n_cl = int(rng.integers(2, 5))
        for _ in range(n_cl * 4):
            if len(clusters) == n_cl:
                break
            fp = _footprint(rng, w, h)
            if fp is None:
                continue
            pads, halo = fp
            layer = 0 if rng.random() < 0.7 else layers - 1
            clusters.append((pads, halo, layer))
        if len(clusters) < 2:  # too small for two footprints: two single pads
            clusters = [([(2, 2)], 1, 0), ([(w - 3, h - 3)], 1, layers - 1)]
        own = {}
        for ci, (pads, halo, layer) in enumerate(clusters):
            xs = [p[0] for p in pads]
            ys = [p[1] for p in pads]
            bx0, bx1 = max(min(xs) - halo - 1, 0), min(max(xs) + halo + 1, w - 1)
            by0, by1 = max(min(ys) - halo - 1, 0), min(max(ys) + halo + 1, h - 1)
            pl = board[layer]
            # courtyard: a step from outside the box into its border is refused
            if bx0 > 0:
                pl[by0:by1 + 1, bx0] |= BOARD_EDGE_NEG_X
            if bx1 < w - 1:
                pl[by0:by1 + 1, bx1] |= BOARD_EDGE_POS_X
            if by0 > 0:
                pl[by0, bx0:bx1 + 1] |= BOARD_EDGE_NEG_Y
            if by1 < h - 1:
                pl[by1, bx0:bx1 + 1] |= BOARD_EDGE_POS_Y
            for (px, py) in pads:
                cost[layer, max(py - halo, 0):py + halo + 1, max(px - halo, 0):px + halo + 1] = OBSTACLE
            if ci < 2:
                px, py = pads[int(rng.integers(0, len(pads)))]
                cells = [dims.idx3(x, y, layer) for y in range(max(py - halo, 0), min(py + halo, h - 1) + 1)
                         for x in range(max(px - halo, 0), min(px + halo, w - 1) + 1)]
                own[ci] = (dims.idx3(px, py, layer), cells)
        src, src_cells = own[0]
        dst, dst_cells = own[1]
        pads_list = sorted(set(src_cells) | set(dst_cells))
        net = NetEndpoints(f"u{k}", src, dst, pads_list)
        grid = Grid(dims, cost.reshape(-1), board.reshape(-1))
        out.append(Workload("uneven", grid, [net], [IsolatedRouteWindow.full(dims)], np.ones(w - 1, np.uint32),
                            np.ones(h - 1, np.uint32), [10] * (layers - 1), None, {}))
    meta = {"workload": f"uneven instances, {n_instances} nets", "seed": seed,
            "side": f"LogNormal(ln {median:g}, sigma {sigma:g}) clamped {lo}-{hi}, per axis",
            "layers": f"uniform {min_layers}-{max_layers}", "pads": "2-4 clusters of 4-40 pads, 1-2 rows, "
            "pitch 2-5, 1-2 cell keepout halo (obstacles), courtyard incoming-edge bits on the pad layer",
            "step": 1, "via": 10, "windows": "whole instance (the net's bounding box)"}
    return InstanceSet("uneven", out, meta)


def snapshot_board(seed: int = 4, w: int = 2048, h: int = 2048, layers: int = 6, n_nets: int = 3000,
                   median: float = 300.0, sigma: float = 0.5, blocked_frac: float = 0.05,
                   via_cost: int = 30) -> Workload:
    """The board of the snapshot negotiation rounds.

    Undirected planar edge prices 10 + Geom(p=0.5) (failures before the first
    success), stored on both in-edge slots; unit enter weights; keepout
    rectangles 8-64 cells a side on random layers until `blocked_frac` of the
    cells are obstacles; via 30.  Two-pin nets: source uniform over free cells,
    Manhattan distance ~ LogNormal(ln median, sigma) clamped to [8, w + h - 2],
    split uniformly between x and y with random signs, target on a random
    layer (redrawn until free); windows by net_window."""
    rng = np.random.default_rng(seed)
    dims = Dims(w, h, layers)
    n = len(dims)
    cost = np.ones((layers, h, w), dtype=np.uint32)
    target = int(blocked_frac * n)
    blocked = 0
    while blocked < target:
        rw, rh = int(rng.integers(8, 65)), int(rng.integers(8, 65))
        x0, y0 = int(rng.integers(0, max(w - rw, 0) + 1)), int(rng.integers(0, max(h - rh, 0) + 1))
        l = int(rng.integers(0, layers))
        sl = cost[l, y0:y0 + rh, x0:x0 + rw]
        blocked += int((sl != OBSTACLE).sum())
        sl[...] = OBSTACLE
    d = np.full((layers, h, w, 4), OBSTACLE, dtype=np.uint32)
    ex = (10 + rng.geometric(0.5, (layers, h, max(w - 1, 0))) - 1).astype(np.uint32)
    ey = (10 + rng.geometric(0.5, (layers, max(h - 1, 0), w)) - 1).astype(np.uint32)
    d[:, :, 1:, 1] = ex  # x -> x+1 enters from -x
    d[:, :, :-1, 2] = ex
    d[:, 1:, :, 0] = ey
    d[:, :-1, :, 3] = ey
    grid = Grid(dims, cost.reshape(-1))
    free = cost.reshape(-1) != OBSTACLE
    nets = []
    while len(nets) < n_nets:
        src = int(rng.integers(0, n))
        if not free[src]:
            continue
        sx, sy, _ = dims.xyz(src)
        dist = int(np.clip(round(median * np.exp(sigma * rng.standard_normal())), 8, w + h - 2))
        dx = int(round(dist * rng.random()))
        dy = dist - dx
        tx = int(np.clip(sx + (dx if rng.random() < 0.5 else -dx), 0, w - 1))
        ty = int(np.clip(sy + (dy if rng.random() < 0.5 else -dy), 0, h - 1))
        dst = dims.idx3(tx, ty, int(rng.integers(0, layers)))
        if not free[dst] or dst == src:
            continue
        nets.append(NetEndpoints(f"s{len(nets)}", src, dst))
    wins = [_net_window(dims, nt) for nt in nets]
    meta = {"workload": f"snapshot negotiation {w}x{h}x{layers}, {n_nets} nets", "seed": seed,
            "edge_price": "10 + Geom(p=0.5) per undirected planar edge, Geom support {0,1,...}",
            "keepouts": f"rectangles 8-64 cells a side, {blocked_frac:.0%} of cells", "via": via_cost,
            "manhattan": f"LogNormal(ln {median:g}, sigma {sigma:g}) clamped [8, w+h-2]", "windows": "net_window"}
    return Workload("snapshot", grid, nets, wins, np.full(w - 1, 10, np.uint32), np.full(h - 1, 10, np.uint32),
                    [via_cost] * (layers - 1), d.reshape(-1), meta)


def serving_pool(seed: int = 5, n_boards: int = 16, lo: int = 64, hi: int = 1024, min_layers: int = 2,
                 max_layers: int = 6) -> List[Workload]:
    """Boards of the serving workload, generated as the congestion board: side
    log-uniform in [lo, hi] (square), layers uniform in [min_layers, max_layers]."""
    rng = np.random.default_rng(seed)
    pool = []
    for k in range(n_boards):
        side = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        layers = int(rng.integers(min_layers, max_layers + 1))
        pool.append(congestion_board(seed=seed * 1000 + k, w=side, h=side, layers=layers, n_nets=0))
    return pool


def serving_trace(pool: List[Workload], rate: float, n_requests: int, seed: int = 6, min_nets: int = 16,
                  max_nets: int = 512):
    """Poisson arrivals at `rate` req/s: (arrival time s, Workload) pairs, each
    a pool board with its own nets (count log-uniform in [min_nets, max_nets])."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        k = int(rng.integers(0, len(pool)))
        b = pool[k]
        n = int(round(np.exp(rng.uniform(np.log(min_nets), np.log(max_nets)))))
        legal = (b.grid.board_constraint & BOARD_TRACE_NODE) == 0
        dims = b.grid.dims
        nets = [NetEndpoints(f"q{i}-{j}", _pick_free(rng, b.grid, dims, legal), _pick_free(rng, b.grid, dims, legal))
                for j in range(n)]
        wins = [_net_window(dims, nt) for nt in nets]
        out.append((t, Workload("serving", b.grid, nets, wins, b.x, b.y, b.vias, b.directed,
                                dict(b.meta, n_nets=n, board_index=k))))
    return out
