"""CPU restatement of one snapshot negotiation round: the test oracle of
mrc_negotiation_round.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the oracle; the product never
imports it.

The round is the reference's Jacobi negotiation iteration
(crates/mr-cpu/src/negotiated.rs:1610-1991) with occupancy and history kept
per directed planar edge slot (the generalisation the engine implements; the
reference counts cells):

* dirty set (:1632-1642): round 0 every net; later, every net with no path or
  whose path uses an edge that two or more nets used after the previous round;
* rip-up of the dirty nets' old paths (:1771-1790);
* frozen snapshot price per slot: base == MAX ? MAX
  : min(base + history + pfac * present_weight * present, MAX - 1), with
  pfac = 1 + round (priced_with_base :2768-2795, passable_search_cost
  :1171-1173);
* each dirty net routed alone on the snapshot by the oracle's astar_buf
  (window, then the full board: :1720-1760);
* merge in net-index order (:1771-1812), then history += history_step on every
  slot whose count is >= 2 (the group overuse scan and history bump,
  :1923-1948, on edges).

Slots per cell are (-y, -x, +x, +y) in-edges; an undirected edge {a, b} counts
at b's slot "from a" and at a's slot "from b".

With connection groups (`groups`, one id per net) the overuse test is the
reference's group-aware scan (:1923-1943): a slot is overused when nets of two
or more distinct groups use it; history, the overused count and the next dirty
set follow it, while prices still count every net's presence.

With a clearance (`clearance` cells of planar halo around every path cell,
`via_keepout` cells around every via; the reference's clearance-active
iteration, :1565-1568 and :1631-1634) the round is the reference's snapshot
branch as written, on slots for copper and on cells for halos:

* every net is routed every round until a round ends without overuse;
* nothing is ripped up before pricing: the snapshot holds every net's previous
  path (present, per slot) and clearance footprint (halo, per cell,
  for_each_halo_cell :3184-3271 on a uniform grid: the (2r+1)^2 box on the
  path cell's own layer, the box of max(clearance, keepout) on both layers of
  every via, base obstacles skipped, counted with multiplicity);
* each net is priced with its own contribution subtracted
  (priced_with_base :2778-2797): base == MAX ? MAX : min(base + history
  + pfac * present_weight * (present - own_path_slot)
  + pfac * halo_weight * (halo - own_halo), MAX - 1);
* the merge then replaces every routed net's old path and footprint by its new
  ones (:1771-1812).
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np

from mrcuda.types import COST_MAX, IsolatedRouteRequest

CAP = COST_MAX - 1


def edge_slots(path: List[int], w: int, plane: int):
    """(cells, slots) arrays of both slots of every planar step of a path."""
    if not path or len(path) < 2:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    p = np.asarray(path, dtype=np.int64)
    a, b = p[:-1], p[1:]
    same = (a // plane) == (b // plane)
    d = b - a
    cells, slots = [], []
    for delta, sb, sa in ((1, 1, 2), (-1, 2, 1), (w, 0, 3), (-w, 3, 0)):
        m = same & (d == delta)
        if delta == 1:
            m &= (a % plane) % w + 1 < w
        elif delta == -1:
            m &= (a % plane) % w > 0
        cells += [b[m], a[m]]
        slots += [np.full(int(m.sum()), sb), np.full(int(m.sum()), sa)]
    return np.concatenate(cells), np.concatenate(slots)


def base_prices(req: IsolatedRouteRequest) -> np.ndarray:
    """Base in-prices (cells, 4): the directed plane, or the per-axis prices."""
    dims = req.grid.dims
    n = len(dims)
    if req.directed_in_costs is not None:
        return np.asarray(req.directed_in_costs, dtype=np.uint32).reshape(n, 4).copy()
    x = np.asarray(req.x_edge_costs, dtype=np.uint32)
    y = np.asarray(req.y_edge_costs, dtype=np.uint32)
    out = np.full((dims.layers, dims.h, dims.w, 4), COST_MAX, dtype=np.uint32)
    if dims.h > 1:
        out[:, 1:, :, 0] = y[:, None]
        out[:, :-1, :, 3] = y[:, None]
    if dims.w > 1:
        out[:, :, 1:, 1] = x[None, :]
        out[:, :, :-1, 2] = x[None, :]
    return out.reshape(n, 4)


def halo_footprint(path, dims, cost: np.ndarray, clearance: int, via_keepout: int) -> np.ndarray:
    """Cells of a path's clearance footprint, with repeats (for_each_halo_cell,
    negotiated.rs:3184-3271, on a uniform grid where a radius of n is the
    n-cell Chebyshev box)."""
    out = []

    def box(x, y, l, r):
        if r <= 0:
            return
        xs = np.arange(max(x - r, 0), min(x + r, dims.w - 1) + 1)
        ys = np.arange(max(y - r, 0), min(y + r, dims.h - 1) + 1)
        c = ((l * dims.h + ys[:, None]) * dims.w + xs[None, :]).reshape(-1)
        out.append(c[cost[c] != COST_MAX])

    if path:
        pts = [dims.xyz(c) for c in path]
        for x, y, l in pts:
            box(x, y, l, clearance)
        vr = max(clearance, via_keepout)
        for (ax, ay, al), (bx, by, bl) in zip(pts, pts[1:]):
            if ax == bx and ay == by and al != bl:
                box(ax, ay, al, vr)
                box(bx, by, bl, vr)
    return np.concatenate(out).astype(np.int64) if out else np.zeros(0, np.int64)


class SnapshotNegotiation:
    def __init__(self, oracle, req: IsolatedRouteRequest, present_weight: int = 16, history_step: int = 1,
                 threads: int = 0, groups=None, clearance: int = 0, via_keepout: int = 0, halo_weight: int = 16):
        self.o = oracle
        self.groups = None if groups is None else [int(g) for g in groups]
        self.req = req
        self.dims = req.grid.dims
        self.weight = int(present_weight)
        self.step = int(history_step)
        self.threads = threads
        n = len(self.dims)
        self.base = base_prices(req)
        self.present = np.zeros((n, 4), dtype=np.uint32)
        self.history = np.zeros((n, 4), dtype=np.uint32)
        self.snapshot = None
        self.paths: List[Optional[List[int]]] = [None] * len(req.nets)
        self.dirty = list(range(len(req.nets)))
        self.round_no = 0
        self.clearance, self.via_keepout = int(clearance), int(via_keepout)
        self.halo_weight = int(halo_weight)
        self.clear = self.clearance > 0 or self.via_keepout > 0
        self.halo = np.zeros(n, dtype=np.uint32)
        self.cost = np.asarray(req.grid.cost, dtype=np.uint32).reshape(-1)

    def _apply(self, path, delta: int):
        c, s = edge_slots(path or [], self.dims.w, self.dims.plane)
        if c.size:
            (np.add if delta > 0 else np.subtract).at(self.present, (c, s), np.uint32(1))
        if self.clear:
            h = halo_footprint(path, self.dims, self.cost, self.clearance, self.via_keepout)
            if h.size:
                (np.add if delta > 0 else np.subtract).at(self.halo, h, np.uint32(1))

    def _price(self, pfac: int, own_slots=None, own_halo=None) -> np.ndarray:
        """Snapshot prices (cells, 4), optionally with one net's own path slots
        and footprint counts subtracted."""
        present = self.present.astype(np.int64)
        halo = self.halo.astype(np.int64)
        if own_slots is not None:
            present = present.copy()
            np.subtract.at(present, own_slots, 1)
        if own_halo is not None and own_halo.size:
            halo = halo.copy()
            np.subtract.at(halo, own_halo, 1)
        price = (self.base.astype(np.uint64) + self.history.astype(np.uint64)
                 + np.uint64(pfac * self.weight) * present.astype(np.uint64)
                 + (np.uint64(pfac * self.halo_weight) * halo.astype(np.uint64))[:, None])
        snap = np.minimum(price, np.uint64(CAP)).astype(np.uint32)
        snap[self.base == COST_MAX] = COST_MAX
        return snap

    def _route_clearance(self, pfac: int, dirty) -> list:
        """Every net in `dirty` routed alone on the snapshot minus its own
        contribution (one oracle call per net: each sees its own prices)."""
        r = self.req
        out = []
        for i in dirty:
            p = self.paths[i]
            own_slots = edge_slots(p, self.dims.w, self.dims.plane) if p else None
            own_halo = halo_footprint(p, self.dims, self.cost, self.clearance, self.via_keepout) if p else None
            price = self._price(pfac, own_slots, own_halo)
            sub = IsolatedRouteRequest(r.grid, [r.nets[i]], [r.windows[i]], r.x_edge_costs, r.y_edge_costs,
                                       r.via_edge_costs, price.reshape(-1))
            paths, _ = self.o.isolated_batch(sub, retry_full=True, mode="astar", threads=self.threads)
            out.append(paths[0])
        return out

    def round(self) -> dict:
        pfac = 1 + self.round_no
        dirty = self.dirty
        stats = {"round": self.round_no, "pfac": pfac, "dirty": len(dirty)}
        if not dirty:
            return stats
        if self.clear:
            self.snapshot = self._price(pfac)
            new_paths = self._route_clearance(pfac, dirty)
            for i, p in zip(dirty, new_paths):  # merge in net-index order: old path and halo out, new ones in
                self._apply(self.paths[i], -1)
                self.paths[i] = p
                self._apply(p, +1)
            return self._settle(stats, dirty)
        for i in dirty:
            self._apply(self.paths[i], -1)
        b = self.base.astype(np.uint64)
        price = b + self.history.astype(np.uint64) + np.uint64(pfac * self.weight) * self.present.astype(np.uint64)
        snap = np.minimum(price, np.uint64(CAP)).astype(np.uint32)
        snap[self.base == COST_MAX] = COST_MAX
        self.snapshot = snap
        r = self.req
        sub = IsolatedRouteRequest(r.grid, [r.nets[i] for i in dirty], [r.windows[i] for i in dirty],
                                   r.x_edge_costs, r.y_edge_costs, r.via_edge_costs, snap.reshape(-1))
        new_paths, _ = self.o.isolated_batch(sub, retry_full=True, mode="astar", threads=self.threads)
        for i, p in zip(dirty, new_paths):  # merge in net-index order
            self.paths[i] = p
            self._apply(p, +1)
        return self._settle(stats, dirty)

    def _settle(self, stats: dict, dirty) -> dict:
        over = self.present >= 2 if self.groups is None else self._group_overuse()
        h = self.history.astype(np.uint64) + over.astype(np.uint64) * np.uint64(self.step)
        self.history = np.minimum(h, np.uint64(COST_MAX)).astype(np.uint32)
        nxt = []
        for i, p in enumerate(self.paths):
            if not p:
                nxt.append(i)
                continue
            c, s = edge_slots(p, self.dims.w, self.dims.plane)
            if c.size and bool(over[c, s].any()):
                nxt.append(i)
        if self.clear:  # every net again until a round without overuse
            nxt = list(range(len(self.paths))) if bool(over.any()) else []
        self.dirty = nxt
        stats.update(routed=sum(1 for i in dirty if self.paths[i]), overused_edges=int(over.sum()) // 2,
                     next_dirty=len(nxt))
        self.round_no += 1
        return stats

    def _group_overuse(self) -> np.ndarray:
        """(cells, 4) flags: slots used by nets of two or more distinct groups."""
        keys, grp = [], []
        for i, p in enumerate(self.paths):
            c, s = edge_slots(p or [], self.dims.w, self.dims.plane)
            keys.append(c * 4 + s)
            grp.append(np.full(c.size, self.groups[i], dtype=np.int64))
        over = np.zeros(self.present.shape, dtype=bool)
        if keys:
            k, g = np.concatenate(keys), np.concatenate(grp)
            pairs = np.unique(np.stack([k, g], axis=1), axis=0) if k.size else np.zeros((0, 2), np.int64)
            uk, cnt = np.unique(pairs[:, 0], return_counts=True)
            over.reshape(-1)[uk[cnt >= 2]] = True
        return over


class SnapshotShard:
    """One shard of the sharded round (the protocol of mrc_negotiation_create_shard):
    it routes only the nets in `owned`, keeps the occupancy of its own paths in
    `local`, and reads the `glob` occupancy that the caller sets to the sum of
    every shard's local occupancy between the phases ripup / route / settle."""

    def __init__(self, oracle, req: IsolatedRouteRequest, owned, present_weight: int = 16, history_step: int = 1):
        self.o = oracle
        self.req = req
        self.dims = req.grid.dims
        self.weight, self.step = int(present_weight), int(history_step)
        n = len(self.dims)
        self.base = base_prices(req)
        self.local = np.zeros((n, 4), dtype=np.uint32)
        self.glob = np.zeros((n, 4), dtype=np.uint32)
        self.history = np.zeros((n, 4), dtype=np.uint32)
        self.owned = [bool(x) for x in owned]
        self.paths: List[Optional[List[int]]] = [None] * len(req.nets)
        self.dirty = [i for i in range(len(req.nets)) if self.owned[i]]
        self.round_no = 0

    def _apply(self, path, delta: int):
        c, s = edge_slots(path or [], self.dims.w, self.dims.plane)
        if c.size:
            (np.add if delta > 0 else np.subtract).at(self.local, (c, s), np.uint32(1))

    def ripup(self):
        for i in self.dirty:
            self._apply(self.paths[i], -1)

    def route(self):
        pfac = 1 + self.round_no
        price = (self.base.astype(np.uint64) + self.history.astype(np.uint64)
                 + np.uint64(pfac * self.weight) * self.glob.astype(np.uint64))
        snap = np.minimum(price, np.uint64(CAP)).astype(np.uint32)
        snap[self.base == COST_MAX] = COST_MAX
        r = self.req
        if self.dirty:
            sub = IsolatedRouteRequest(r.grid, [r.nets[i] for i in self.dirty], [r.windows[i] for i in self.dirty],
                                       r.x_edge_costs, r.y_edge_costs, r.via_edge_costs, snap.reshape(-1))
            new_paths, _ = self.o.isolated_batch(sub, retry_full=True, mode="astar")
            for i, p in zip(self.dirty, new_paths):
                self.paths[i] = p
                self._apply(p, +1)

    def settle(self):
        over = self.glob >= 2
        h = self.history.astype(np.uint64) + over.astype(np.uint64) * np.uint64(self.step)
        self.history = np.minimum(h, np.uint64(COST_MAX)).astype(np.uint32)
        nxt = []
        for i, p in enumerate(self.paths):
            if not self.owned[i]:
                continue
            if not p:
                nxt.append(i)
                continue
            c, s = edge_slots(p, self.dims.w, self.dims.plane)
            if c.size and bool((self.glob[c, s] >= 2).any()):
                nxt.append(i)
        self.dirty = nxt
        self.round_no += 1
        return int(over.sum()) // 2
