"""Plain data types mirroring metalroute's contract crate and provider seam.

These are the Python-side shapes of the C ABI in ``include/mr_cuda.h``; they
carry no routing logic.  Field names and meanings follow the reference:

* ``Dims`` / ``Grid`` / ``NetEndpoints`` — crates/mr-core/src/lib.rs:40-165,
  394-513, 519-537 (row-major ``idx3(x, y, l) = (l*h + y)*w + x``,
  ``OBSTACLE = 0xFFFFFFFF``, ``Grid::BOARD_*`` mask bits).
* ``IsolatedRouteWindow`` / ``IsolatedRouteRequest`` —
  crates/mr-cpu/src/negotiated.rs:489-537.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

OBSTACLE = 0xFFFFFFFF
COST_MAX = 0xFFFFFFFF

BOARD_TRACE_NODE = 1 << 0
BOARD_VIA_NODE = 1 << 1
BOARD_EDGE_NEG_Y = 1 << 2
BOARD_EDGE_NEG_X = 1 << 3
BOARD_EDGE_POS_X = 1 << 4
BOARD_EDGE_POS_Y = 1 << 5


@dataclass(frozen=True)
class Dims:
    w: int
    h: int
    layers: int = 1

    def __len__(self) -> int:
        return self.w * self.h * self.layers

    @property
    def plane(self) -> int:
        return self.w * self.h

    def idx(self, x: int, y: int) -> int:
        return y * self.w + x

    def idx3(self, x: int, y: int, layer: int) -> int:
        return (layer * self.h + y) * self.w + x

    def xyz(self, i: int):
        layer, r = divmod(i, self.w * self.h)
        return r % self.w, r // self.w, layer

    def xy(self, i: int):
        r = i % (self.w * self.h)
        return r % self.w, r // self.w


@dataclass
class Grid:
    dims: Dims
    cost: np.ndarray
    board_constraint: Optional[np.ndarray] = None
    via_forbidden: Optional[np.ndarray] = None

    @staticmethod
    def filled(dims: Dims, fill: int) -> "Grid":
        return Grid(dims, np.full(len(dims), fill, dtype=np.uint32))

    def __post_init__(self):
        self.cost = np.ascontiguousarray(self.cost, dtype=np.uint32)
        if self.board_constraint is not None:
            self.board_constraint = np.ascontiguousarray(self.board_constraint, dtype=np.uint8)
        if self.via_forbidden is not None:
            self.via_forbidden = np.ascontiguousarray(self.via_forbidden, dtype=np.uint8)

    def is_obstacle(self, i: int) -> bool:
        return int(self.cost[i]) == OBSTACLE

    def set(self, i: int, c: int) -> None:
        self.cost[i] = c


@dataclass
class NetEndpoints:
    net: str
    src: int
    dst: int
    passable_pads: List[int] = field(default_factory=list)
    via_passable_pads: List[int] = field(default_factory=list)


@dataclass(frozen=True)
class IsolatedRouteWindow:
    x0: int
    y0: int
    x1: int
    y1: int

    @staticmethod
    def full(dims: Dims) -> "IsolatedRouteWindow":
        return IsolatedRouteWindow(0, 0, max(dims.w - 1, 0), max(dims.h - 1, 0))

    def contains(self, dims: Dims, cell: int) -> bool:
        x, y = dims.xy(cell)
        return self.x0 <= x <= self.x1 and self.y0 <= y <= self.y1

    def cells(self, dims: Dims) -> int:
        return (self.x1 - self.x0 + 1) * (self.y1 - self.y0 + 1) * dims.layers


@dataclass
class IsolatedRouteRequest:
    """Borrowed static inputs of one isolated batch (negotiated.rs:521-537).

    ``directed_in_costs`` is the engine's superset form: 4 base prices per cell
    for the planar in-edges from the -y, -x, +x, +y neighbours, with
    0xFFFFFFFF marking a blocked edge.  When given it replaces the per-axis gap
    price; the destination enter weight and the 0xFFFFFFFE step cap still apply.
    """

    grid: Grid
    nets: Sequence[NetEndpoints]
    windows: Sequence[IsolatedRouteWindow]
    x_edge_costs: Sequence[int]
    y_edge_costs: Sequence[int]
    via_edge_costs: Sequence[Optional[int]]
    directed_in_costs: Optional[np.ndarray] = None


def group_of(name: str) -> str:
    """A net's connection-group name: the prefix before the first '#'
    (negotiated.rs:915-922)."""
    i = name.find("#")
    return name if i < 0 else name[:i]


def connection_group_ids(nets: Sequence[NetEndpoints]) -> List[int]:
    """Dense connection-group ids, the reference's connection_group_ids
    (negotiated.rs:929-989): nets whose names share a group_of prefix, or that
    share an endpoint cell, are one group (union toward the lower index); ids
    are numbered by the first appearance of each group's root."""
    n = len(nets)
    parent = list(range(n))

    def find(x: int) -> int:
        root = x
        while parent[root] != root:
            root = parent[root]
        while parent[x] != root:
            parent[x], x = root, parent[x]
        return root

    def union(a: int, b: int) -> None:
        ra, rb = find(a), find(b)
        if ra != rb:
            if ra < rb:
                parent[rb] = ra
            else:
                parent[ra] = rb

    by_name: Dict[str, int] = {}
    for i, nt in enumerate(nets):
        j = by_name.setdefault(group_of(nt.net), i)
        if j != i:
            union(i, j)
    by_cell: Dict[int, int] = {}
    for i, nt in enumerate(nets):
        for c in (nt.src, nt.dst):
            j = by_cell.setdefault(c, i)
            if j != i:
                union(i, j)
    ids: Dict[int, int] = {}
    return [ids.setdefault(find(i), len(ids)) for i in range(n)]
